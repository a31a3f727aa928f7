// Image segmentation pyramid (SegHAC with LabelISPFormat, target 1):
// reference segment.cu:1279-1321. The path runs CentroidLink, 4-neighbour
// grid, sigma = 0; Min / Max / Ward linkage, the 8-neighbour grid and the
// Gaussian pre-blur are the reference's other configurations.
//
// Level l holds N_l nodes and E_l directed edges. Per level the loop runs
// CRTrees on the 1-NN successor array, records the level in the reference's
// ISP layout (segment.cu:884-905), then builds level l+1:
//   * edges mapped to parents, sorted as (s, t) pairs, de-duplicated and
//     stripped of self-loops; boundary lengths are summed by POSITION in the
//     sorted order, because the reference sorts the pairs alone and leaves the
//     length array in its old order (segment.cu:1061, :368-386);
//   * inner distance max of the children (segment.cu:1116-1128);
//   * child sums of (L, a, b, x, y, count), added in increasing child index
//     (the reference uses float atomics, segment.cu:472-486);
//   * centroid distance with the hinge on L, fused as the reference's device
//     code fuses it (Ward: times w_s w_t / (w_s + w_t), :559-577), or for
//     Min / Max linkage the min / max of the merged edges' distances
//     (reduce_dist, :336-366), plus the penalty d += max(d - maxinner[t], 0)
//     (segment.cu:508-534, :582-612);
//   * per node the minimum over its out-edges, ties to the largest target
//     (segment.cu:403-422, :1211-1231).
#include <algorithm>

#include "engine.h"

namespace hbp
{
namespace
{
__device__ __forceinline__ float pix_dist(float4 s, float4 t)
{
    float dx = s.x - t.x, dy = s.y - t.y, dz = s.z - t.z;
    float d = __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
    return __fadd_rn(d, dx > 0.f ? dx : 0.f);
}

// compute_1nn_grid_k (segment.cu:57-195), NB = 4 or 8: neighbours up, down,
// left, right, then up-left, up-right, down-right, down-left; first strict
// minimum. Also writes the level-0 edge list bd[NB*i+k] = (i, neighbour or i),
// the edge distances (edist, Min / Max linkage only; 0 on self-edges) and the
// level-0 sums (L, a, b, x, y, w).
template <int NB>
__global__ void nn_grid_kernel(const float4 *__restrict__ lab, int W, int H, int *__restrict__ nn,
                               float *__restrict__ dist_min, int2 *__restrict__ bd,
                               int *__restrict__ bdl, float *__restrict__ sums, float *__restrict__ edist)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = W * H;
    if (i >= n)
        return;
    int y = i / W, x = i - y * W;
    float4 s = lab[i];
    const bool up = y > 0, dn = y < H - 1, lf = x > 0, rt = x < W - 1;
    int nb[8] = {up ? i - W : -1,           dn ? i + W : -1,           lf ? i - 1 : -1,
                 rt ? i + 1 : -1,           up && lf ? i - W - 1 : -1, up && rt ? i - W + 1 : -1,
                 dn && rt ? i + W + 1 : -1, dn && lf ? i + W - 1 : -1};
    float best = 3.402823466e+38f;
    int arg = 0;
#pragma unroll
    for (int k = 0; k < NB; ++k)
    {
        int t = nb[k];
        bd[NB * i + k] = make_int2(i, t < 0 ? i : t);
        bdl[NB * i + k] = 1;
        if (edist)
            edist[NB * i + k] = 0.0f;
        if (t < 0)
            continue;
        float d = pix_dist(s, lab[t]);
        if (edist)
            edist[NB * i + k] = d;
        if (d < best)
        {
            best = d;
            arg = t;
        }
    }
    nn[i] = arg;
    dist_min[i] = best;
    if (sums)
    {
        sums[i] = s.x;
        sums[n + i] = s.y;
        sums[2 * n + i] = s.z;
        sums[3 * n + i] = (float)x;
        sums[4 * n + i] = (float)y;
        sums[5 * n + i] = s.w;
    }
}

__global__ void map_edges(const int2 *__restrict__ bd, const int *__restrict__ clus, long E, int bits,
                          uint64_t *__restrict__ keys)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E)
        return;
    int2 v = bd[e];
    keys[e] = ((uint64_t)(uint32_t)clus[v.x] << bits) | (uint32_t)clus[v.y];
}

__global__ void run_flags(const uint64_t *__restrict__ keys, long E, int bits, int *__restrict__ keep)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E)
        return;
    uint64_t k = keys[e];
    uint32_t s = (uint32_t)(k >> bits), t = (uint32_t)(k & ((1ull << bits) - 1));
    bool last = (e == E - 1) || keys[e + 1] != k;
    keep[e] = (last && s != t) ? 1 : 0;
}

// Kept run ends become the new edges; every non-self-loop element adds the
// length stored at its sorted POSITION into its run's slot (integer atomics:
// the order does not matter).
__global__ void emit_edges(const uint64_t *__restrict__ keys, const int *__restrict__ keep,
                           const int *__restrict__ slot, const int *__restrict__ bdl_old, long E,
                           int bits, int2 *__restrict__ bd_new, int *__restrict__ bdl_new)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E)
        return;
    uint64_t k = keys[e];
    int s = (int)(k >> bits), t = (int)(k & ((1ull << bits) - 1));
    if (s == t)
        return;
    int sl = slot[e];
    atomicAdd(&bdl_new[sl], bdl_old[e]);
    if (keep[e])
        bd_new[sl] = make_int2(s, t);
}

__global__ void iota_u32(uint32_t *v, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        v[i] = (uint32_t)i;
}

__global__ void copy_keys(const int *clus, int n, uint32_t *k, int *count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        k[i] = (uint32_t)clus[i];
        atomicAdd(&count[clus[i]], 1);
    }
}

// Per parent: sums of the children (children in increasing index, sequential
// from 0) and the maximum of the children's dist_min (inner distance).
__global__ void parent_sums(const uint32_t *__restrict__ child, const int *__restrict__ child_off,
                            const float *__restrict__ sums_c, int Nc, const float *__restrict__ dmin_c,
                            int Np, float *__restrict__ sums_p, float *__restrict__ dmax_p,
                            float *__restrict__ mean_p)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Np)
        return;
    int b = child_off[p], e = child_off[p + 1];
    float acc[6] = {0, 0, 0, 0, 0, 0};
    float mx = 0.0f;
    for (int j = b; j < e; ++j)
    {
        int c = (int)child[j];
#pragma unroll
        for (int ch = 0; ch < 6; ++ch)
            acc[ch] = __fadd_rn(acc[ch], sums_c[(size_t)ch * Nc + c]);
        mx = fmaxf(mx, dmin_c[c]);
    }
#pragma unroll
    for (int ch = 0; ch < 6; ++ch)
        sums_p[(size_t)ch * Np + p] = acc[ch];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
        mean_p[(size_t)ch * Np + p] = __fdiv_rn(acc[ch], acc[5]);
    dmax_p[p] = mx;
}

// reduce_dist (segment.cu:336-366) for Min / Max linkage: every merged edge
// (s, t), s != t, folds its distance into the new edge (s, t) with min / max.
// The new edges are sorted by (s, t), so t is found by binary search in s's
// out-edge range. Distances are >= 0, so their bit patterns order as ints.
__global__ void reduce_edge_dist(const int2 *__restrict__ bd_c, const float *__restrict__ edist_c,
                                 const int *__restrict__ clus, long E, const int2 *__restrict__ bd_p,
                                 const int *__restrict__ off_p, int use_max, float *__restrict__ edist_p)
{
    long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E)
        return;
    const int2 v = bd_c[e];
    const int s = clus[v.x], t = clus[v.y];
    if (s == t)
        return;
    int lo = off_p[s], hi = off_p[s + 1] - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if (bd_p[mid].y < t)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo > hi || bd_p[lo].y != t)
        return; // cannot happen: every merged pair is a new edge
    int *dst = reinterpret_cast<int *>(edist_p + lo);
    const int bits = __float_as_int(edist_c[e]);
    if (use_max)
        atomicMax(dst, bits);
    else
        atomicMin(dst, bits);
}

__global__ void fill_f32(float *p, long n, float v)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        p[i] = v;
}

__global__ void edge_src_count(const int2 *__restrict__ bd, int E, int *__restrict__ count)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < E)
        atomicAdd(&count[bd[e].x], 1);
}

// One thread per node walks its out-edges (contiguous, targets ascending):
// the edge distance (centroid from the means, times the Ward weight from the
// weight sums wsum; or the reduced distance in edist for Min / Max, where the
// penalised value is written back for the next level) + penalty, minimum, and
// the largest target among minima.
__global__ void node_1nn(const int2 *__restrict__ bd, const int *__restrict__ off, int N,
                         const float *__restrict__ mean, const float *__restrict__ dmax,
                         int *__restrict__ nn, float *__restrict__ dist_min, int link,
                         const float *__restrict__ wsum, float *__restrict__ edist)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N)
        return;
    float ls = mean[s], as = mean[N + s], bs = mean[2 * N + s];
    float best = 3.402823466e+38f;
    int arg = 0;
    for (int e = off[s]; e < off[s + 1]; ++e)
    {
        int t = bd[e].y;
        float d;
        if (link == LINK_MIN || link == LINK_MAX)
            d = edist[e];
        else
        {
            float e0 = __fsub_rn(ls, mean[t]), e1 = __fsub_rn(as, mean[N + t]), e2 = __fsub_rn(bs, mean[2 * N + t]);
            float h = e0 > 0.f ? e0 : 0.f;
            d = __fmaf_rn(e2, e2, __fmaf_rn(e1, e1, __fmaf_rn(e0, e0, h)));
            if (link == LINK_WARD)
            {
                const float sw = wsum[s], tw = wsum[t];
                d = __fmul_rn(__fdiv_rn(__fmul_rn(sw, tw), __fadd_rn(sw, tw)), d);
            }
        }
        float delta = __fsub_rn(d, dmax[t]);
        if (delta > 0)
            d = __fadd_rn(d, delta);
        if (edist)
            edist[e] = d;
        if (d < best)
        {
            best = d;
            arg = t;
        }
        else if (d == best)
            arg = t;
    }
    nn[s] = arg;
    dist_min[s] = best;
}

// ---------------------------------------------------------------------------
// SegHAC::get_target_clus (segment.cu:1016-1041) with compute_dist_pos,
// compute_scaned_pos, set_pre_clus_label and reset_clus_label (:635-755,
// :954-1014): the Nn clusters CRTrees just formed from N nodes (Nn <= target
// < N) become exactly `target`. Clusters are ranked by the sum of their
// children's 1-NN distances, largest first (a stable descending sort, ties to
// the lower label); ranks 0..b, b the first rank where breaking ranks 0..b
// yields at least target clusters, are broken into their children, which take
// the labels cum(i)-1, cum(i)-2, ... (cum: inclusive sum of the ranked child
// counts) in increasing child index, capped at exact = target - Nn + b (the
// children past the cap stay merged); unbroken rank i takes i + target - Nn.
// Fixed orders where the reference has none: the distance sums add children
// in increasing index (float atomics there) and the children of a broken
// cluster take their labels in increasing index (atomicSub order there).

// Per cluster c (children val[off[c] ..] in increasing index): the distance
// sum as a descending sort key (the sums are >= 0, so the complemented bits
// order them largest first) and c as its value.
__global__ void target_sums(const uint32_t *val, const int *off, const float *dmin, int Nn, uint32_t *key,
                            uint32_t *lab)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nn)
        return;
    float s = 0.0f;
    for (int j = off[c]; j < off[c + 1]; ++j)
        s = s + dmin[val[j]];
    key[c] = ~__float_as_uint(s);
    lab[c] = (uint32_t)c;
}

// child count of the cluster ranked i (cnt[Nn] = 0 for the scan's total)
__global__ void target_counts(const uint32_t *lab, const int *off, int Nn, int *cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Nn)
        cnt[i] = off[lab[i] + 1] - off[lab[i]];
    else if (i == Nn)
        cnt[Nn] = 0;
}

// is_break_cluster: the first rank b with cum(b) + Nn - b - 1 >= target
// (cum(i) = ex[i + 1]; the count is non-decreasing in i)
__global__ void target_break(const int *ex, int Nn, int target, int *b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < Nn && ex[i + 1] + Nn - i - 1 >= target)
        atomicMin(b, i);
}

__global__ void target_assign(const uint32_t *lab, const int *off, const uint32_t *val, const int *ex,
                              const int *bptr, int Nn, int target, int *clus)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Nn)
        return;
    const int b = *bptr, exact = target - Nn + b, c = (int)lab[i];
    const int j0 = off[c], j1 = off[c + 1];
    for (int j = j0; j < j1; ++j)
        clus[val[j]] = i <= b ? min(ex[i + 1] - 1 - (j - j0), exact) : i + target - Nn;
}

int bits_for(long n)
{
    int b = 1;
    while ((1l << b) < n)
        ++b;
    return b;
}

int read_int(const int *dev, cudaStream_t st)
{
    int h = 0;
    HBP_CUDA(cudaMemcpyAsync(&h, dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    HBP_CUDA(cudaStreamSynchronize(st));
    return h;
}

// get_target_clus on the labels clus (N nodes -> Nn clusters, Nn < target < N)
// with the nodes' 1-NN distances dmin: clus then holds labels 0..target-1.
void target_relabel(int *clus, const float *dmin, int N, int Nn, int target, Arena &tmp, cudaStream_t st)
{
    size_t m = tmp.mark();
    uint32_t *ck = tmp.alloc<uint32_t>(N), *ck_alt = tmp.alloc<uint32_t>(N);
    uint32_t *val = tmp.alloc<uint32_t>(N), *val_alt = tmp.alloc<uint32_t>(N);
    int *count = tmp.alloc<int>(Nn + 1), *off = tmp.alloc<int>(Nn + 1);
    uint32_t *key = tmp.alloc<uint32_t>(Nn), *key_alt = tmp.alloc<uint32_t>(Nn);
    uint32_t *lab = tmp.alloc<uint32_t>(Nn), *lab_alt = tmp.alloc<uint32_t>(Nn);
    int *ex = tmp.alloc<int>(Nn + 1), *b = tmp.alloc<int>(1);
    // the children of every cluster in increasing index
    HBP_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (Nn + 1), st));
    copy_keys<<<ceil_div(N, 256), 256, 0, st>>>(clus, N, ck, count);
    note_launch();
    iota_u32<<<ceil_div(N, 256), 256, 0, st>>>(val, N);
    note_launch();
    HBP_LAUNCH_CHECK();
    radix_sort_pairs_u32(ck, val, ck_alt, val_alt, N, bits_for(Nn), tmp, st);
    exclusive_scan(count, off, Nn + 1, nullptr, tmp, st);
    // rank by distance sum, then the cumulative child counts in rank order
    target_sums<<<ceil_div(Nn, 128), 128, 0, st>>>(val, off, dmin, Nn, key, lab);
    note_launch();
    HBP_LAUNCH_CHECK();
    radix_sort_pairs_u32(key, lab, key_alt, lab_alt, Nn, 32, tmp, st);
    target_counts<<<ceil_div(Nn + 1, 128), 128, 0, st>>>(lab, off, Nn, count);
    note_launch();
    HBP_LAUNCH_CHECK();
    exclusive_scan(count, ex, Nn + 1, nullptr, tmp, st);
    HBP_CUDA(cudaMemsetAsync(b, 0x7f, sizeof(int), st)); // 0x7f7f7f7f: above every rank
    target_break<<<ceil_div(Nn, 128), 128, 0, st>>>(ex, Nn, target, b);
    note_launch();
    target_assign<<<ceil_div(Nn, 128), 128, 0, st>>>(lab, off, val, ex, b, Nn, target, clus);
    note_launch();
    HBP_LAUNCH_CHECK();
    tmp.rewind(m);
}
} // namespace

namespace
{
// update_image_label through levels 0..L-1 (segment.cu:871-883): a pixel's
// label is clus_{L-1}(...clus_0(px)), its cluster after level L-1.
__global__ void top_labels(const int *clus, const long *node_off, int L, int n, int *labels)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int v = i;
    for (int l = 0; l < L; ++l)
        v = clus[node_off[l] + v];
    labels[i] = v;
}

__global__ void max_label(const int *clus, int n, int *mx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        atomicMax(mx, clus[i]);
}

// draw_segmentation's three pictures of a label image (segment.cu:907-951,
// kernels :213-292): label+1 as a BGR byte triple (low byte first), label+1
// as an int, or the input image with the pixels whose left or upper
// neighbour lies in another cluster painted red (0,0,255).
__global__ void draw_labels(const int *labels, const uint8_t *bgr, int W, int H, int format, void *out)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W)
        return;
    const int i = y * W + x, c = labels[i];
    if (format == SEG_DRAW_INT)
    {
        static_cast<int *>(out)[i] = c + 1;
        return;
    }
    uint8_t *o = static_cast<uint8_t *>(out) + 3 * (size_t)i;
    if (format == SEG_DRAW_UCHAR3)
    {
        const unsigned v = (unsigned)(c + 1);
        o[0] = (uint8_t)v;
        o[1] = (uint8_t)(v >> 8);
        o[2] = (uint8_t)(v >> 16);
        return;
    }
    const bool edge = (x > 0 && labels[i - 1] != c) || (y > 0 && labels[i - W] != c);
    const uint8_t *s = bgr + 3 * (size_t)i;
    o[0] = edge ? 0 : s[0];
    o[1] = edge ? 0 : s[1];
    o[2] = edge ? 255 : s[2];
}
} // namespace

void launch_draw_segmentation(const Pyramid &pyr, int level, int format, const uint8_t *bgr, void *out,
                              Arena &tmp, cudaStream_t st)
{
    size_t m = tmp.mark();
    int *labels = tmp.alloc<int>((size_t)pyr.W * pyr.H);
    launch_level_labels(pyr, level, labels, tmp, st);
    draw_labels<<<dim3(ceil_div(pyr.W, 128), pyr.H), 128, 0, st>>>(labels, bgr, pyr.W, pyr.H, format, out);
    note_launch();
    HBP_LAUNCH_CHECK();
    HBP_CUDA(cudaStreamSynchronize(st));
    tmp.rewind(m);
}

void launch_level_labels(const Pyramid &pyr, int level, int *labels, Arena &tmp, cudaStream_t st)
{
    // the level offsets as a small device array (the pageable copy is staged
    // before cudaMemcpyAsync returns)
    std::vector<long> off(pyr.node_off.begin(), pyr.node_off.end());
    size_t m = tmp.mark();
    long *doff = tmp.alloc<long>(off.size());
    HBP_CUDA(cudaMemcpyAsync(doff, off.data(), sizeof(long) * off.size(), cudaMemcpyHostToDevice, st));
    const int n = pyr.W * pyr.H;
    top_labels<<<ceil_div(n, 256), 256, 0, st>>>(pyr.clus, doff, level + 1, n, labels);
    note_launch();
    HBP_LAUNCH_CHECK();
    HBP_CUDA(cudaStreamSynchronize(st));
    tmp.rewind(m);
}

int level_cluster_count(const Pyramid &pyr, int level, Arena &tmp, cudaStream_t st)
{
    if (level + 1 < pyr.L)
        return pyr.N[level + 1];
    size_t m = tmp.mark();
    int *mx = tmp.alloc<int>(1);
    HBP_CUDA(cudaMemsetAsync(mx, 0, sizeof(int), st));
    const int top = pyr.L - 1;
    max_label<<<ceil_div(pyr.N[top], 256), 256, 0, st>>>(pyr.clus + pyr.node_off[top], pyr.N[top], mx);
    note_launch();
    HBP_LAUNCH_CHECK();
    const int h = read_int(mx, st);
    tmp.rewind(m);
    return h + 1;
}

void check_seg_config(const SegConfig &cfg)
{
    if (cfg.link < LINK_MIN || cfg.link > LINK_WARD)
        throw StatusError{HBP_ERR_INVALID_ARG, "linkage must be 0 (Min), 1 (Max), 2 (Centroid) or 3 (Ward)"};
    if (cfg.num_nb != 4 && cfg.num_nb != 8)
        throw StatusError{HBP_ERR_INVALID_ARG, "num_nb must be 4 or 8"};
    if (!(cfg.sigma >= 0.0) || blur_radius(cfg.sigma) > BLUR_MAX_S)
        throw StatusError{HBP_ERR_INVALID_ARG, "sigma must lie in [0, 2.5): the blur radius round(3 sigma) <= 7"};
    if (cfg.target < 1)
        throw StatusError{HBP_ERR_INVALID_ARG, "target_clus must be >= 1"};
}

void segment_image(const uint8_t *bgr, int W, int H, Pyramid &pyr, Arena &a, Arena &tmp,
                   int *err_dev, cudaStream_t st, const SegConfig &cfg)
{
    check_seg_config(cfg);
    const int N0 = W * H, NB = cfg.num_nb;
    if (cfg.target >= N0)
        throw StatusError{HBP_ERR_INVALID_ARG, "target_clus must be below the pixel count"};
    const bool use_mean = cfg.link == LINK_CENTROID || cfg.link == LINK_WARD;
    pyr.W = W;
    pyr.H = H;
    pyr.L = 0;
    pyr.N.clear();
    pyr.E.clear();
    pyr.node_off.clear();
    pyr.edge_off.clear();
    pyr.child_base.clear();
    pyr.nb_base.clear();
    // capacities of the concatenated ISP arrays (segment.hpp:276-283)
    pyr.clus = a.alloc<int>(2 * (size_t)N0);
    pyr.sums = a.alloc<float>(12 * (size_t)N0);
    pyr.bd = a.alloc<int2>(2 * (size_t)NB * N0);
    pyr.bdl = a.alloc<int>(2 * (size_t)NB * N0);
    pyr.child = a.alloc<uint32_t>(2 * (size_t)N0);
    pyr.child_off = a.alloc<int>(2 * (size_t)N0 + 64);
    pyr.nb_off = a.alloc<int>(2 * (size_t)N0 + 64);

    size_t m0 = tmp.mark();
    float4 *lab = tmp.alloc<float4>(N0);
    int *nn = tmp.alloc<int>(N0), *nn2 = tmp.alloc<int>(N0);
    float *dmin = tmp.alloc<float>(N0), *dmin2 = tmp.alloc<float>(N0);
    float *mean = tmp.alloc<float>(3 * (size_t)N0);
    float *dmax = tmp.alloc<float>(N0);
    int *count = tmp.alloc<int>(N0 + 1);
    int *num_dev = tmp.alloc<int>(2);
    uint64_t *keys = tmp.alloc<uint64_t>((size_t)NB * N0), *keys_alt = tmp.alloc<uint64_t>((size_t)NB * N0);
    int *keep = tmp.alloc<int>((size_t)NB * N0), *slot = tmp.alloc<int>((size_t)NB * N0);
    uint32_t *ck = tmp.alloc<uint32_t>(N0), *ck_alt = tmp.alloc<uint32_t>(N0),
             *cv_alt = tmp.alloc<uint32_t>(N0);
    // edge distances of the current and the next level (Min / Max linkage)
    float *edist = use_mean ? nullptr : tmp.alloc<float>((size_t)NB * N0);
    float *edist2 = use_mean ? nullptr : tmp.alloc<float>((size_t)NB * N0);

    if (cfg.sigma > 1.1754943508222875e-38) // FLT_MIN, as segment.cu:805
    {
        size_t mb = tmp.mark();
        float4 *blur = tmp.alloc<float4>(N0);
        launch_lab_blur(bgr, W, H, cfg.sigma, blur, lab, st);
        tmp.rewind(mb); // later users of the scratch run after the blur (same stream)
    }
    else
        launch_lab(bgr, N0, lab, st);
    if (NB == 8)
        nn_grid_kernel<8><<<ceil_div(N0, 256), 256, 0, st>>>(lab, W, H, nn, dmin, pyr.bd, pyr.bdl, pyr.sums, edist);
    else
        nn_grid_kernel<4><<<ceil_div(N0, 256), 256, 0, st>>>(lab, W, H, nn, dmin, pyr.bd, pyr.bdl, pyr.sums, edist);
    note_launch();
    HBP_LAUNCH_CHECK();

    int N = N0;
    long E = (long)NB * N0;
    size_t oc = 0, ob = 0, och = 0, onb = 0;
    for (;;)
    {
        int *clus = pyr.clus + oc;
        crtrees_labels(nn, N, clus, num_dev, err_dev, tmp, st);
        int Nn = read_int(num_dev, st);
        if (Nn < 1 || Nn > N)
            throw StatusError{HBP_ERR_NO_CONVERGENCE, "crtrees produced an invalid cluster count"};
        if (Nn < cfg.target) // N > target: the previous level stopped above it
        {
            target_relabel(clus, dmin, N, Nn, cfg.target, tmp, st);
            Nn = cfg.target;
        }
        pyr.N.push_back(N);
        pyr.E.push_back((int)E);
        pyr.node_off.push_back(oc);
        pyr.edge_off.push_back(ob);
        pyr.L++;
        // children of every parent in increasing child index; used for the
        // sums here and by the spatial propagation of HBP (sort_clus,
        // hbp_isp.cu:985-1001)
        uint32_t *child = pyr.child + oc;
        int *child_off = pyr.child_off + och;
        pyr.child_base.push_back(och);
        HBP_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (Nn + 1), st));
        copy_keys<<<ceil_div(N, 256), 256, 0, st>>>(clus, N, ck, count);
        note_launch();
        iota_u32<<<ceil_div(N, 256), 256, 0, st>>>(child, N);
        note_launch();
        HBP_LAUNCH_CHECK();
        radix_sort_pairs_u32(ck, child, ck_alt, cv_alt, N, bits_for(Nn), tmp, st);
        exclusive_scan(count, child_off, Nn + 1, nullptr, tmp, st);
        och += Nn + 1;
        // CSR by source of this level's edges (sorted by source at every level)
        int *nb_off = pyr.nb_off + onb;
        pyr.nb_base.push_back(onb);
        HBP_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (N + 1), st));
        edge_src_count<<<ceil_div(E, 256), 256, 0, st>>>(pyr.bd + ob, (int)E, count);
        note_launch();
        HBP_LAUNCH_CHECK();
        exclusive_scan(count, nb_off, N + 1, nullptr, tmp, st);
        onb += N + 1;
        if (Nn == cfg.target) // 1: the pyramid up to one node
            break;

        // next level's nodes and edges live right after this level's
        float *sums_c = pyr.sums + 6 * oc;
        float *sums_p = pyr.sums + 6 * (oc + N);
        int2 *bd_c = pyr.bd + ob;
        int *bdl_c = pyr.bdl + ob;
        int2 *bd_p = pyr.bd + ob + E;
        int *bdl_p = pyr.bdl + ob + E;
        // reduce_boundary_dist
        int bits = bits_for(Nn);
        map_edges<<<ceil_div(E, 256), 256, 0, st>>>(bd_c, clus, E, bits, keys);
        note_launch();
        HBP_LAUNCH_CHECK();
        radix_sort_keys_u64(keys, keys_alt, E, 2 * bits, tmp, st);
        run_flags<<<ceil_div(E, 256), 256, 0, st>>>(keys, E, bits, keep);
        note_launch();
        HBP_LAUNCH_CHECK();
        exclusive_scan(keep, slot, E, num_dev + 1, tmp, st);
        int E2 = read_int(num_dev + 1, st);
        if ((size_t)(ob + E + E2) > 2 * (size_t)NB * N0 || E2 < 1)
            throw StatusError{HBP_ERR_INTERNAL, "edge capacity exceeded"};
        HBP_CUDA(cudaMemsetAsync(bdl_p, 0, sizeof(int) * E2, st));
        emit_edges<<<ceil_div(E, 256), 256, 0, st>>>(keys, keep, slot, bdl_c, E, bits, bd_p, bdl_p);
        note_launch();
        HBP_LAUNCH_CHECK();
        // sums, means, inner max (reduce_data_mean, compute_dist_inner_max)
        parent_sums<<<ceil_div(Nn, 128), 128, 0, st>>>(child, child_off, sums_c, N, dmin, Nn, sums_p,
                                                         dmax, mean);
        note_launch();
        HBP_LAUNCH_CHECK();
        // CSR of the new edges for the per-node minimum
        HBP_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * (Nn + 1), st));
        edge_src_count<<<ceil_div(E2, 256), 256, 0, st>>>(bd_p, E2, count);
        note_launch();
        HBP_LAUNCH_CHECK();
        exclusive_scan(count, slot, Nn + 1, nullptr, tmp, st);
        if (!use_mean)
        {
            fill_f32<<<ceil_div(E2, 256), 256, 0, st>>>(edist2, E2, cfg.link == LINK_MIN ? 3.402823466e+38f : 0.0f);
            note_launch();
            reduce_edge_dist<<<ceil_div(E, 256), 256, 0, st>>>(bd_c, edist, clus, E, bd_p, slot,
                                                               cfg.link == LINK_MAX ? 1 : 0, edist2);
            note_launch();
            HBP_LAUNCH_CHECK();
        }
        node_1nn<<<ceil_div(Nn, 128), 128, 0, st>>>(bd_p, slot, Nn, mean, dmax, nn2, dmin2, cfg.link,
                                                     sums_p + 5 * (size_t)Nn, edist2);
        note_launch();
        HBP_LAUNCH_CHECK();
        std::swap(nn, nn2);
        std::swap(dmin, dmin2);
        std::swap(edist, edist2);
        oc += N;
        ob += E;
        N = Nn;
        E = E2;
        if (oc + N > 2 * (size_t)N0)
            throw StatusError{HBP_ERR_INTERNAL, "node capacity exceeded"};
    }
    tmp.rewind(m0);
}

} // namespace hbp
