// CPU oracle, segmentation pyramid (test infrastructure; see oracle_common.h).
#include <algorithm>
#include <cfloat>
#include <numeric>

#include "oracle_api.h"
#include "oracle_common.h"

using namespace orc;

namespace
{
int find(std::vector<int> &p, int x)
{
    while (p[x] != x)
    {
        p[x] = p[p[x]];
        x = p[x];
    }
    return x;
}

// Canonical form of CRTrees::get_clus (CRTrees.cu:315-354). In a functional
// graph every weakly connected component holds exactly one cycle. The
// reference de-links every node whose in-degree (counted from the still
// active nodes) exceeds one, pointer-jumps the others onto those roots and
// re-links the roots to the next root along their original successor; the
// roots become the active set of the next round (R_1 = in-degree > 1 in the
// input, R_{t+1} = in-degree > 1 among R_t in the contracted graph). A
// component stops once its active set forms a cycle (no in-degree > 1 left);
// a component that never had such a node is a plain cycle. Every node then
// points straight at a node of that final cycle, and the max-pointer-jumping
// of CRTrees.cu:170-187/274-297 labels the whole component with the largest
// node index on the final cycle.
void crtrees_labels(const int *nn, int N, std::vector<int> &label)
{
    label.assign(N, -1);
    std::vector<int> uf(N);
    std::iota(uf.begin(), uf.end(), 0);
    for (int i = 0; i < N; ++i)
    {
        int a = find(uf, i), b = find(uf, nn[i]);
        if (a != b)
            uf[a] = b;
    }
    std::vector<int> comp(N);
    for (int i = 0; i < N; ++i)
        comp[i] = find(uf, i);

    std::vector<int> indeg(N, 0);
    for (int i = 0; i < N; ++i)
        indeg[nn[i]]++;
    std::vector<char> inR(N, 0), compHasR(N, 0);
    std::vector<int> R;
    for (int i = 0; i < N; ++i)
        if (indeg[i] > 1)
        {
            inR[i] = 1;
            R.push_back(i);
            compHasR[comp[i]] = 1;
        }
    // plain cycles: label = max node of the component (all nodes are on the cycle)
    std::vector<int> compMax(N, -1);
    for (int i = 0; i < N; ++i)
        if (!compHasR[comp[i]])
            compMax[comp[i]] = std::max(compMax[comp[i]], i);

    // next root reached from each node following the successor (memoised)
    std::vector<int> root(N, -1);
    std::vector<int> stack;
    auto root_of = [&](int j, const int *succ, const std::vector<char> &in) {
        stack.clear();
        while (!in[j] && root[j] < 0)
        {
            stack.push_back(j);
            j = succ[j];
        }
        int r = in[j] ? j : root[j];
        for (int k : stack)
            root[k] = r;
        return r;
    };
    std::vector<int> next(N, -1);
    for (int r : R)
        next[r] = root_of(nn[r], nn, inR);

    std::vector<char> done(N, 0);
    while (!R.empty())
    {
        std::vector<int> deg(N, 0);
        for (int r : R)
            deg[next[r]]++;
        std::vector<char> compCont(N, 0);
        for (int r : R)
            if (deg[r] > 1)
                compCont[comp[r]] = 1;
        std::vector<int> R2;
        std::vector<char> inR2(N, 0);
        for (int r : R)
        {
            if (!compCont[comp[r]])
            {
                // this component's active set is its final cycle
                compMax[comp[r]] = std::max(compMax[comp[r]], r);
                continue;
            }
            if (deg[r] > 1)
            {
                R2.push_back(r);
                inR2[r] = 1;
            }
        }
        // contracted successor: first R2 node on next, next(next), ...
        std::fill(root.begin(), root.end(), -1);
        std::vector<int> next2(N, -1);
        for (int r : R2)
            next2[r] = root_of(next[r], next.data(), inR2);
        R.swap(R2);
        next.swap(next2);
    }
    for (int i = 0; i < N; ++i)
        label[i] = compMax[comp[i]];
}

int compact_labels(std::vector<int> &label, int N)
{
    std::vector<int> used(N, 0);
    for (int i = 0; i < N; ++i)
        used[label[i]] = 1;
    std::vector<int> pos(N, 0);
    int k = 0;
    for (int i = 0; i < N; ++i)
    {
        pos[i] = k;
        k += used[i];
    }
    for (int i = 0; i < N; ++i)
        label[i] = pos[label[i]];
    return k;
}
} // namespace

extern "C" {

// CRTrees::get_clus + compact_clus_label (CRTrees.cu:315-354, :387-403):
// component labels in 0..n-1, ordered by each component's label value.
int orc_crtrees(const int *nn, int N, int *clus)
{
    std::vector<int> lab;
    crtrees_labels(nn, N, lab);
    int k = compact_labels(lab, N);
    std::copy(lab.begin(), lab.end(), clus);
    return k;
}

// Kernel-by-kernel simulation of CRTrees::get_clus (CRTrees.cu:28-354) with
// the reference's ping-pong buffers, each kernel reading the state before it
// (re_link's in-place reads, CRTrees.cu:98-120, take the pre-kernel value).
// Used only to cross-check orc_crtrees.
int orc_crtrees_literal(const int *nn_in, int N, int *clus_out)
{
    std::vector<int> nn(nn_in, nn_in + N), save(nn), C(nn), Nb(N, 0), mask(N, 1), maskc(N),
        indeg(N);
    for (;;)
    {
        std::fill(indeg.begin(), indeg.end(), 0);
        for (int i = 0; i < N; ++i)
            if (mask[i])
                indeg[C[i]]++;
        bool more = false;
        for (int i = 0; i < N; ++i)
            if (mask[i] && indeg[i] > 1)
                more = true;
        if (!more)
            break;
        maskc = mask;
        std::fill(mask.begin(), mask.end(), 0);
        for (int i = 0; i < N; ++i)
            if (indeg[i] > 1)
            {
                C[i] = i;
                mask[i] = 1;
            }
        // pointer_jumping: odd rounds write Nb from C, even rounds C from Nb;
        // the caller keeps reading C.
        std::vector<int> *cur = &C, *oth = &Nb;
        bool flag = true;
        while (flag)
        {
            flag = false;
            for (int i = 0; i < N; ++i)
            {
                if (!maskc[i])
                    continue;
                int a = (*cur)[i], b = (*cur)[a];
                (*oth)[i] = b;
                if (!mask[a] && mask[b])
                    flag = true;
            }
            std::swap(cur, oth);
        }
        std::vector<int> old(C);
        for (int i = 0; i < N; ++i)
        {
            if (mask[i])
            {
                int v = nn[i];
                C[i] = mask[v] ? v : old[v];
            }
            else if (!maskc[i])
            {
                int n = old[i];
                if (maskc[n])
                    C[i] = old[n];
            }
        }
        for (int i = 0; i < N; ++i)
        {
            int v = C[i];
            if (mask[i])
                nn[i] = v;
            else if (mask[v])
                nn[i] = C[v];
        }
        C = nn;
    }
    nn = save;
    // pointer_jumping_max (CRTrees.cu:274-297)
    std::vector<int> M(C), K(N, 0);
    std::vector<int> *cn = &C, *on = &Nb, *cm = &M, *om = &K;
    bool flag = true;
    while (flag)
    {
        flag = false;
        for (int i = 0; i < N; ++i)
        {
            int a = (*cn)[i];
            int m = std::max((*cm)[i], (*cm)[a]);
            (*om)[i] = m;
            (*on)[i] = (*cn)[a];
            if (m != (*cm)[i])
                flag = true;
        }
        std::swap(cn, on);
        std::swap(cm, om);
    }
    std::vector<int> lab(K);
    int k = compact_labels(lab, N);
    std::copy(lab.begin(), lab.end(), clus_out);
    return k;
}

// SegHAC::get_target_clus (segment.cu:1016-1041) with compute_dist_pos,
// compute_scaned_pos, set_pre_clus_label and reset_clus_label (:635-755,
// :954-1014): the num clusters that CRTrees just formed from num_p nodes
// (num <= target < num_p) are ranked by the sum of their children's 1-NN
// distances, largest first (ties: lower label first; the reference's sort is
// a stable descending radix sort). The first b+1 ranked clusters are broken
// into their children, b the first rank where breaking ranks 0..b gives at
// least target clusters; the children of broken rank i take the labels
// cum(i)-1, cum(i)-2, ... (cum: inclusive sum of the ranked child counts) in
// increasing child index, every label above exact = target - num + b becomes
// exact (those children stay merged), and unbroken rank i takes
// i + target - num. The labels are then 0 .. target-1. Fixed orders where the
// reference has none: the distance sums add children in increasing index
// (float atomics there), and the children of a broken cluster take their
// labels in increasing index (atomicSub order there).
static int target_clusters(std::vector<int> &clus, const std::vector<float> &dist_min, int num_p, int num, int target)
{
    if (num == target)
        return num;
    std::vector<float> dist(num, 0.0f);
    std::vector<int> cnt(num, 0);
    for (int i = 0; i < num_p; ++i)
    {
        dist[clus[i]] += dist_min[i];
        cnt[clus[i]]++;
    }
    std::vector<int> order(num);
    for (int c = 0; c < num; ++c)
        order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return dist[a] > dist[b]; });
    std::vector<int> cum(num), rank(num);
    for (int i = 0; i < num; ++i)
    {
        cum[i] = (i ? cum[i - 1] : 0) + cnt[order[i]];
        rank[order[i]] = i;
    }
    int b = num - 1;
    for (int i = 0; i < num; ++i)
        if (cum[i] + num - i - 1 >= target)
        {
            b = i;
            break;
        }
    const int exact = target - num + b;
    std::vector<int> used(num, 0);
    for (int k = 0; k < num_p; ++k)
    {
        const int i = rank[clus[k]];
        if (i <= b)
            clus[k] = std::min(cum[i] - 1 - used[clus[k]]++, exact);
        else
            clus[k] = i + target - num;
    }
    return target;
}

// SegHAC::run_ms with LabelISPFormat (segment.cu:1279-1321), for
// the linkages of segment.hpp:8-16 (0 Min, 1 Max, 2 Centroid, 3 Ward) and a
// 4- or 8-neighbour pixel grid. Input: LAB float4 image (its fourth channel is
// the pixel weight). Output: the image segmentation pyramid in the reference's
// ISP layout (segment.cu:884-905): per level l, num_clus N_l and num_bd E_l
// (level_sizes[2l], [2l+1]); clus (N_l ints: node -> parent), mean (6 x N_l
// floats, channel-major: sums of L, a, b, x, y and the weight), bd (E_l int
// pairs), bdl (E_l ints), concatenated over levels. Capacities: clus 2*HW,
// mean 12*HW, bd 4*num_nb*HW ints, bdl 2*num_nb*HW. Returns the number of
// levels. target: SegHAC's target_clus; 1 builds the pyramid up to one
// node, target > 1 (below W*H) stops at the first level whose CRTrees pass
// leaves at most target clusters, after get_target_clus made them exactly
// target: that level's clus maps its nodes to the target superpixels.
//
// Child sums are added in increasing child index starting from 0.0f (the
// reference adds them with float atomics in an unspecified order,
// segment.cu:472-486).
int orc_segment_target(const float *lab4, int W, int H, int link, int num_nb, int target, int max_levels,
                       int *level_sizes, int *clus_out, float *mean_out, int *bd_out, int *bdl_out)
{
    if (link < 0 || link > 3 || (num_nb != 4 && num_nb != 8) || target < 1 || target >= W * H)
        return -1;
    const bool use_mean = link == 2 || link == 3; // segment.hpp:248
    const int N0 = W * H;
    std::vector<int> nn(N0), bd(2 * (size_t)num_nb * N0), bdl((size_t)num_nb * N0, 1);
    std::vector<float> dist_min(N0), sums(6 * (size_t)N0), edist((size_t)num_nb * N0);
    orc_nn_grid_nb(lab4, W, H, num_nb, nn.data(), dist_min.data(), bd.data(), edist.data());
    for (int i = 0; i < N0; ++i)
    {
        sums[i] = lab4[4 * (size_t)i];
        sums[(size_t)N0 + i] = lab4[4 * (size_t)i + 1];
        sums[2 * (size_t)N0 + i] = lab4[4 * (size_t)i + 2];
        sums[3 * (size_t)N0 + i] = (float)(i % W);
        sums[4 * (size_t)N0 + i] = (float)(i / W);
        sums[5 * (size_t)N0 + i] = lab4[4 * (size_t)i + 3];
    }
    int num = N0, E = num_nb * N0, levels = 0;
    size_t oc = 0, ob = 0;
    std::vector<int> clus;
    for (;;)
    {
        clus.resize(num);
        int num_new = orc_crtrees(nn.data(), num, clus.data());
        if (num_new <= target)
            num_new = target_clusters(clus, dist_min, num, num_new, target);
        // push the level (segment.cu:884-905)
        if (levels < max_levels)
        {
            level_sizes[2 * levels] = num;
            level_sizes[2 * levels + 1] = E;
        }
        std::copy(clus.begin(), clus.end(), clus_out + oc);
        std::copy(sums.begin(), sums.begin() + 6 * (size_t)num, mean_out + 6 * oc);
        std::copy(bd.begin(), bd.begin() + 2 * (size_t)E, bd_out + 2 * ob);
        std::copy(bdl.begin(), bdl.begin() + E, bdl_out + ob);
        oc += num;
        ob += E;
        levels++;
        if (num_new == target)
            break;

        // reduce_boundary_dist (segment.cu:1050-1091): map edges to parents,
        // sort the (s, t) pairs, keep the last of each run unless it is a
        // self-loop; boundary lengths are summed by POSITION in the sorted
        // order (the bdl array is not permuted with the pairs, :1061,
        // :368-386). Min / Max linkage carry each edge's distance through the
        // sort and reduce each run with min / max (reduce_dist, :336-366),
        // which no order changes.
        std::vector<std::pair<uint64_t, float>> key(E);
        for (int e = 0; e < E; ++e)
        {
            uint32_t s = (uint32_t)clus[bd[2 * (size_t)e]], t = (uint32_t)clus[bd[2 * (size_t)e + 1]];
            key[e] = {((uint64_t)s << 32) | t, edist[e]};
        }
        std::sort(key.begin(), key.end(),
                  [](const std::pair<uint64_t, float> &a, const std::pair<uint64_t, float> &b) { return a.first < b.first; });
        std::vector<int> bd2, bdl2;
        std::vector<float> edist2;
        bd2.reserve(2 * (size_t)E);
        int run_sum = 0;
        float run_d = link == 0 ? FLT_MAX : 0.0f;
        for (int e = 0; e < E; ++e)
        {
            uint32_t s = (uint32_t)(key[e].first >> 32), t = (uint32_t)key[e].first;
            if (s != t)
            {
                run_sum += bdl[e];
                run_d = link == 0 ? std::min(run_d, key[e].second) : std::max(run_d, key[e].second);
            }
            bool last = (e == E - 1) || key[e + 1].first != key[e].first;
            if (last)
            {
                if (s != t)
                {
                    bd2.push_back((int)s);
                    bd2.push_back((int)t);
                    bdl2.push_back(run_sum);
                    edist2.push_back(run_d);
                }
                run_sum = 0;
                run_d = link == 0 ? FLT_MAX : 0.0f;
            }
        }
        int E2 = (int)bdl2.size();

        // compute_dist_inner_max (segment.cu:1116-1128)
        std::vector<float> dmax(num_new, 0.0f);
        for (int c = 0; c < num; ++c)
            dmax[clus[c]] = std::max(dmax[clus[c]], dist_min[c]);
        // reduce_data_mean (segment.cu:1134-1153): child sums in child order;
        // means of channels 0-4, the weight sum stays (sum_to_mean, :492-503)
        std::vector<float> sums2(6 * (size_t)num_new, 0.0f);
        for (int ch = 0; ch < 6; ++ch)
            for (int c = 0; c < num; ++c)
                sums2[(size_t)ch * num_new + clus[c]] += sums[(size_t)ch * num + c];
        std::vector<float> mean2(5 * (size_t)num_new);
        for (int ch = 0; ch < 5; ++ch)
            for (int p = 0; p < num_new; ++p)
                mean2[(size_t)ch * num_new + p] = sums2[(size_t)ch * num_new + p] / sums2[5 * (size_t)num_new + p];
        // compute_dist_mean_k (+ ward_weight, :559-577) or the reduced
        // distance, then pernalize_dist_k and compute_1nn (segment.cu:508-534,
        // :582-612, :1211-1231, :403-422); the centroid distance is fused the
        // way the reference's device code fuses it.
        std::vector<float> dmin2(num_new, FLT_MAX);
        for (int e = 0; e < E2; ++e)
        {
            int s = bd2[2 * (size_t)e], t = bd2[2 * (size_t)e + 1];
            float d;
            if (use_mean)
            {
                float e0 = mean2[s] - mean2[t];
                float e1 = mean2[(size_t)num_new + s] - mean2[(size_t)num_new + t];
                float e2 = mean2[2 * (size_t)num_new + s] - mean2[2 * (size_t)num_new + t];
                float h = e0 > 0.f ? e0 : 0.f;
                d = std::fma(e2, e2, std::fma(e1, e1, std::fma(e0, e0, h)));
                if (link == 3)
                {
                    const float sw = sums2[5 * (size_t)num_new + s], tw = sums2[5 * (size_t)num_new + t];
                    d = sw * tw / (sw + tw) * d;
                }
            }
            else
                d = edist2[e];
            float delta = d - dmax[t];
            if (delta > 0)
                d += delta;
            edist2[e] = d;
            dmin2[s] = std::min(dmin2[s], d);
        }
        std::vector<int> nn2(num_new, 0);
        for (int e = 0; e < E2; ++e)
        {
            int s = bd2[2 * (size_t)e], t = bd2[2 * (size_t)e + 1];
            if (edist2[e] == dmin2[s])
                nn2[s] = std::max(nn2[s], t);
        }
        num = num_new;
        E = E2;
        nn.swap(nn2);
        dist_min.swap(dmin2);
        sums.swap(sums2);
        bd.swap(bd2);
        bdl.swap(bdl2);
        edist.swap(edist2);
    }
    return levels;
}

int orc_segment_cfg(const float *lab4, int W, int H, int link, int num_nb, int max_levels, int *level_sizes,
                    int *clus_out, float *mean_out, int *bd_out, int *bdl_out)
{
    return orc_segment_target(lab4, W, H, link, num_nb, 1, max_levels, level_sizes, clus_out, mean_out, bd_out,
                              bdl_out);
}

// SegHAC::run_ms with CentroidLink and the 4-neighbour grid (the path's
// configuration); see orc_segment_cfg.
int orc_segment(const float *lab4, int W, int H, int max_levels, int *level_sizes, int *clus_out,
                float *mean_out, int *bd_out, int *bdl_out)
{
    return orc_segment_cfg(lab4, W, H, 2, 4, max_levels, level_sizes, clus_out, mean_out, bd_out, bdl_out);
}

} // extern "C"
