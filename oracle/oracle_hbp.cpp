// CPU oracle, hierarchical belief propagation on the segmentation pyramid
// (test infrastructure; see oracle_common.h). Restates HBP_ISP
// (hbp_isp.hpp:122-442, hbp_isp.cu) for one view.
//
// Two modes share the code: R = float reproduces the engine bit for bit
// (same operation order, same reductions); R = double is the FP64 oracle used
// for the message-error report and as the CPU baseline.
//
// Reduction orders fixed by the engine (the reference uses float atomics and
// Thrust reduce_by_key, whose order is unspecified):
//   plane cost of node n, candidate k, over the level's pixel list (sorted by
//   node, raster order inside a node; list positions are absolute), cut into
//   256-position chunks:
//   S0 a chunk the node fills entirely: slot j = positions j, j+32, ...,
//      j+224 added in order, the 32 slots combined by the xor butterfly of
//      orc::butterfly32 (offsets 16..1); other chunks by S1 and S2:
//   S1 the node's positions inside one 32-position window are summed by a
//      Hillis-Steele inclusive scan (off = 1..16: x[r] = x[r-off] + x[r] for
//      r >= off), taking its last element;
//   S2 the S1 pieces inside one 256-position window are added in order;
//   S3 the 256-window sums are added in order.
//   belief[k][s] = cost[k][s] + msg_t of s's out-edges in edge order.
//   dc colour term: (|dL| + |da|) + |db|; position term: dx*dx + dy*dy.
// Smoothness points: the lower-index node's three points, then the other's
// (the reference takes the source's first; the order only moves roundings).
// Fused multiply-adds (the reference's nvcc build contracts these expressions,
// in an order its output does not pin down; HBP agreement with it is the same
// for every order tried): data cost d = fma(a, x, fma(b, y, c)) and
// cost = fma(d + 1 - d_f, V[d], (d_f - d) * V[d+1]); each plane's value at a
// smoothness point fma(a, X, fma(b, Y, c)) and message fma(c0, phi, msg).
// The smoothness term of two planes is sum_i |v_s,i - v_t,i| over the six
// points (the reference evaluates the difference plane at each point,
// hbp_isp.cu:339-344: the same quantity with other roundings), and
// min(phi / 3 / dist_pos, tau_smooth) is taken as min(phi * rq, tau_smooth)
// with rq = (1/3) / dist_pos rounded once per edge (:349, two divisions per
// label there).
#include <algorithm>
#include <cfloat>
#include <cstdio>

#include "oracle_api.h"
#include "oracle_common.h"

using namespace orc;

namespace
{
constexpr int P = 4, K = 12;
constexpr int CHUNK = 256;

template <typename R>
struct P4
{
    R x, y, z, w;
};

template <typename R>
struct Level
{
    int N = 0, E = 0, Nh = 1;
    const int *clus = nullptr; // N -> parent
    std::vector<float> mean;   // 6 x N (means for c < 5, count in c = 5)
    const int *bd = nullptr;   // E pairs
    const int *bdl = nullptr;  // E
    std::vector<int> pix;      // HW pixel ids sorted by (node, pixel)
    std::vector<int> pix_off;  // N + 1
    std::vector<int> nb_off;   // N + 1 (CSR by source)
    std::vector<int> rev;      // E
    std::vector<R> dc;         // 2 x E
    std::vector<int> child;    // N children sorted by (parent, child)
    std::vector<int> child_off; // Nh + 1
    std::vector<P4<R>> plane; // K x N
    std::vector<R> cost, belief; // K x N
    std::vector<int> pid;     // 3 x N
};

// Lock-step shadow (shadow = true): a second copy of the continuous BP state
// (costs, beliefs, messages) in type S, advanced with the main run's discrete
// decisions: the same candidate planes (RANSAC points, spatial picks, random
// adjustments) and the same kept slots (ranks of the main run's beliefs). The
// shadow's messages are compared with the main run's at every BP step; with
// S = double that is the main run's message error against FP64, with S = R
// the shadow repeats the main run exactly (the replay's own check).
template <typename R, typename S = double>
struct Engine
{
    int W, H, D, L;
    R lambda, tau, tau_smooth;
    const uint8_t *vol;           // D x HW (Census: uint8 costs)
    const float *volf = nullptr;  // or floats (MC-CNN); used when set
    const float *wta;
    std::vector<Level<R>> lv;
    std::vector<R> msg, msg_t;
    std::vector<uint32_t> s_child, s_nb, s_ransac;
    std::vector<int> order;
    std::vector<P4<R>> plane_buf;
    long steps = 0, max_steps = -1;
    bool stopped = false;
    bool fp16_msg = false; // messages stored as FP16 (float mode only)
    bool shadow = false;
    std::vector<std::vector<S>> sh_cost, sh_belief; // per level, K x N
    std::vector<S> sh_msg, sh_msg_t;
    // message error: shift-invariant (each message minus its own minimum, in
    // both runs: a per-message constant moves every belief of a node alike and
    // changes no decision) and raw (as stored, each run normalised by the mode)
    double err_max = 0, err_sum = 0, ref_abs_sum = 0, ref_abs_max = 0, raw_max = 0, raw_sum = 0;
    long err_n = 0;

    // read_plane_cost (hbp_isp.cu:205-227) of one pixel, evaluated in T
    template <typename T>
    T pixel_cost(int px, const P4<R> &pl) const
    {
        T x = (T)(px % W), y = (T)(px / W);
        T d_f = std::fma((T)pl.x, x, std::fma((T)pl.y, y, (T)pl.z));
        int d = f2i_rd((float)d_f);
        if (sizeof(T) == 8)
        {
            // FP64 mode: floor in double with the same NaN/saturation rules
            double v = (double)d_f;
            d = v != v ? 0 : (v >= 2147483648.0 ? 2147483647 : (v < -2147483648.0 ? (-2147483647 - 1) : (int)std::floor(v)));
        }
        T cost;
        if (d < 0 || d >= D - 1)
            cost = (T)tau;
        else
        {
            const size_t n = (size_t)W * H;
            T v0, v1;
            if (volf)
            {
                v0 = (T)volf[(size_t)d * n + px];
                v1 = (T)volf[(size_t)(d + 1) * n + px];
            }
            else
            {
                v0 = (T)vol[(size_t)d * n + px];
                v1 = (T)vol[(size_t)(d + 1) * n + px];
            }
            cost = std::fma((T)(d + 1) - d_f, v0, (d_f - (T)d) * v1);
        }
        return (T)lambda * cost;
    }

    // compute_plane_cost (hbp_isp.cu:1159-1174) for slots s_c .. s_c+3, in T,
    // into out (K x N).
    template <typename T>
    void plane_cost_t(const Level<R> &l, int s_c, T *out) const
    {
#pragma omp parallel for schedule(dynamic, 64)
        for (int n = 0; n < l.N; ++n)
        {
            int b = l.pix_off[n], m = l.pix_off[n + 1] - b;
            for (int p = 0; p < P; ++p)
            {
                const P4<R> pl = l.plane[(size_t)(s_c + p) * l.N + n];
                const int e = b + m;
                T total = 0;
                for (int w256 = b / CHUNK; w256 <= (e - 1) / CHUNK; ++w256)
                {
                    const int lo = std::max(b, w256 * CHUNK), hi = std::min(e, (w256 + 1) * CHUNK);
                    T acc = 0;
                    if (lo == w256 * CHUNK && hi == (w256 + 1) * CHUNK)
                    {
                        // the node fills the chunk: slot j sums positions
                        // j, j+32, ..., j+224 in order; xor butterfly
                        T slots[32];
                        for (int j = 0; j < 32; ++j)
                        {
                            T a = pixel_cost<T>(l.pix[lo + j], pl);
                            for (int k = 1; k < CHUNK / 32; ++k)
                                a = a + pixel_cost<T>(l.pix[lo + j + 32 * k], pl);
                            slots[j] = a;
                        }
                        acc = butterfly32(slots);
                        total = w256 == b / CHUNK ? acc : total + acc;
                        continue;
                    }
                    for (int w32 = lo / 32; w32 <= (hi - 1) / 32; ++w32)
                    {
                        const int l2 = std::max(lo, w32 * 32), h2 = std::min(hi, (w32 + 1) * 32);
                        T x[32];
                        for (int q = l2; q < h2; ++q)
                            x[q - l2] = pixel_cost<T>(l.pix[q], pl);
                        const T piece = scan_last(x, h2 - l2);
                        acc = w32 == lo / 32 ? piece : acc + piece;
                    }
                    total = w256 == b / CHUNK ? acc : total + acc;
                }
                out[(size_t)(s_c + p) * l.N + n] = total;
            }
        }
    }
    int level_of(const Level<R> &l) const { return (int)(&l - lv.data()); }
    // the main run's costs of slots s_c .. s_c+3, and the shadow's
    void plane_cost(Level<R> &l, int s_c)
    {
        plane_cost_t<R>(l, s_c, l.cost.data());
        if (shadow)
            plane_cost_t<S>(l, s_c, sh_cost[(size_t)level_of(l)].data());
    }

    // ransac_candidate_plane + make_three_diff_id + fit_plane_from_points
    // (hbp_isp.cu:504-548, :592-640).
    void ransac(Level<R> &l)
    {
#pragma omp parallel for schedule(static)
        for (int n = 0; n < l.N; ++n)
        {
            int cn = l.pix_off[n + 1] - l.pix_off[n], cp = l.pix_off[n];
            uint32_t s = s_ransac[n];
            for (int p = 2 * P; p < 3 * P; ++p)
            {
                s = lcg(s);
                int p0 = (int)(s % (uint32_t)cn);
                s = lcg(s);
                int p1 = cn > 1 ? (int)(s % (uint32_t)(cn - 1)) : 0;
                s = lcg(s);
                int p2 = cn > 2 ? (int)(s % (uint32_t)(cn - 2)) : 0;
                if (cn <= 3)
                {
                    p1 = (p0 + 1) % cn;
                    p2 = (p1 + 1) % cn;
                }
                else
                {
                    if (p1 == p0)
                        p1 = cn - 1;
                    if (p2 == p0)
                        p2 = (p1 == cn - 2) ? cn - 1 : cn - 2;
                    else if (p2 == p1)
                        p2 = (p0 == cn - 2) ? cn - 1 : cn - 2;
                }
                int ids[3] = {l.pix[cp + p0], l.pix[cp + p1], l.pix[cp + p2]};
                R Ax = (R)(ids[0] % W), Ay = (R)(ids[0] / W), Az = (R)wta[ids[0]];
                R Bx = (R)(ids[1] % W), By = (R)(ids[1] / W), Bz = (R)wta[ids[1]];
                R Cx = (R)(ids[2] % W), Cy = (R)(ids[2] / W), Cz = (R)wta[ids[2]];
                R ax = Bx - Ax, ay = By - Ay, az = Bz - Az;
                R bx = Cx - Ax, by = Cy - Ay, bz = Cz - Az;
                R nx = ay * bz - az * by;
                R ny = az * bx - ax * bz;
                R nz = ax * by - ay * bx;
                nx /= nz;
                ny /= nz;
                nz /= nz;
                P4<R> pl;
                R eps = sizeof(R) == 4 ? (R)FLT_EPSILON : (R)DBL_EPSILON;
                if (std::fabs(nz - (R)1) > eps)
                    pl = {0, 0, (Az + Bz + Cz) / (R)3, 0};
                else
                    pl = {-nx, -ny, nx * Ax + ny * Ay + Az, 0};
                l.plane[(size_t)p * l.N + n] = pl;
                if (p == 3 * P - 1)
                {
                    l.pid[3 * (size_t)n] = ids[0];
                    l.pid[3 * (size_t)n + 1] = ids[1];
                    l.pid[3 * (size_t)n + 2] = ids[2];
                }
            }
            s_ransac[n] = s;
        }
    }

    // select_child_plane, neighbor_candidate_plane, set_candidate_plane_k
    // (hbp_isp.cu:676-741, :1225-1243).
    void spatial(int li)
    {
        Level<R> &l = lv[li], &h = lv[li + 1];
        for (int id = 0; id < h.N; ++id)
        {
            int cn = l.child_off[id + 1] - l.child_off[id], cp = l.child_off[id];
            uint32_t s = s_child[id];
            for (int p = 0; p < P; ++p)
            {
                s = lcg(s);
                int c = l.child[cp + (int)(s % (uint32_t)cn)];
                h.plane[(size_t)(p + 2 * P) * h.N + id] = l.plane[c];
            }
            s_child[id] = s;
        }
        for (int id = 0; id < h.N; ++id)
        {
            int nbn = h.nb_off[id + 1] - h.nb_off[id], nbp = h.nb_off[id];
            uint32_t s = s_nb[id];
            for (int p = 0; p < P; ++p)
            {
                s = lcg(s);
                int t = h.bd[2 * (size_t)(nbp + (int)(s % (uint32_t)nbn)) + 1];
                plane_buf[(size_t)p * h.N + id] = h.plane[(size_t)(p + 2 * P) * h.N + t];
            }
            s_nb[id] = s;
        }
        for (int p = 0; p < P; ++p)
            for (int id = 0; id < h.N; ++id)
                h.plane[(size_t)(p + 2 * P) * h.N + id] = plane_buf[(size_t)p * h.N + id];
        for (int n = 0; n < l.N; ++n)
            for (int p = 2 * P; p < 3 * P; ++p)
                l.plane[(size_t)p * l.N + n] = h.plane[(size_t)p * h.N + l.clus[n]];
    }

    // random_candidate_plane + normalize_plane (hbp_isp.cu:495-503, :641-674).
    void random_adjust(Level<R> &l, R max_dz, R max_dn)
    {
        for (int n = 0; n < l.N; ++n)
        {
            uint32_t s = s_ransac[n];
            R x = (R)l.mean[3 * (size_t)l.N + n], y = (R)l.mean[4 * (size_t)l.N + n];
            for (int p = 2 * P; p < 3 * P; ++p)
            {
                P4<R> pl = l.plane[(size_t)p * l.N + n];
                R z = pl.x * x + pl.y * y + pl.z;
                auto unif = [&](R f) {
                    s = lcg(s);
                    return (R)s / (R)2147483648.0 * f;
                };
                R dz = unif(max_dz);
                z += dz;
                R dnx = unif(max_dn), dny = unif(max_dn), dnz = unif(max_dn);
                R norm = std::sqrt(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z);
                pl.x /= norm;
                pl.y /= norm;
                pl.z /= norm;
                pl.x += dnx;
                pl.y += dny;
                pl.z += dnz;
                R a = -pl.x / pl.z, b = -pl.y / pl.z;
                R c = z - a * x - b * y;
                l.plane[(size_t)p * l.N + n] = {a, b, c, 0};
            }
            s_ransac[n] = s;
        }
    }

    // passing_msg_k (hbp_isp.cu:292-304): msg = belief of the target - msg,
    // for the 2P best and prior slots.
    template <typename T>
    void passing_t(const Level<R> &l, const T *belief, T *m) const
    {
        const int N = l.N, E = l.E;
        for (int e = 0; e < E; ++e)
        {
            int t = l.bd[2 * (size_t)e + 1];
            for (int p = 0; p < 2 * P; ++p)
                m[(size_t)p * E + e] = belief[(size_t)p * N + t] - m[(size_t)p * E + e];
        }
    }

    // smooth_msg_k + normalize_msg_k (hbp_isp.cu:273-290, :306-355) in T:
    // msg_t[y][e] = sum over the two groups of min_p msg[p][e] + c0 * phi,
    // normalised by the mean (min_norm = false) or by the minimum, then
    // rounded to FP16 when fp16_store.
    template <typename T>
    void smooth_t(const Level<R> &l, const T *m_in, T *m_out, bool min_norm, bool fp16_store) const
    {
        const int N = l.N, E = l.E;
#pragma omp parallel for schedule(static)
        for (int e = 0; e < E; ++e)
        {
            int s = l.bd[2 * (size_t)e], t = l.bd[2 * (size_t)e + 1];
            // the six points in a fixed order for both directions of an edge:
            // the lower-index node's three, then the other's
            const int lo = std::min(s, t), hi = std::max(s, t);
            T X[6], Y[6];
            for (int i = 0; i < 3; ++i)
            {
                int a = l.pid[3 * (size_t)lo + i], b = l.pid[3 * (size_t)hi + i];
                X[i] = (T)(a % W);
                Y[i] = (T)(a / W);
                X[3 + i] = (T)(b % W);
                Y[3 + i] = (T)(b / W);
            }
            T dist_color = std::fmax((T)l.dc[e], (T)0.01f);
            T dist_pos = std::fmax((T)l.dc[(size_t)E + e], (T)1.0f);
            T c0 = dist_color * (T)l.bdl[e];
            // (phi / 3) / dist_pos as phi times one per-edge factor
            const T rq = ((T)1 / (T)3) / dist_pos;
            // each plane's value at the six points, v = fma(a, X, fma(b, Y, c));
            // phi = sum_i |vs_i - vt_i| in point order
            T vt[2 * P][6];
            for (int p = 0; p < 2 * P; ++p)
            {
                const P4<R> pt = l.plane[(size_t)p * N + t];
                for (int i = 0; i < 6; ++i)
                    vt[p][i] = std::fma((T)pt.x, X[i], std::fma((T)pt.y, Y[i], (T)pt.z));
            }
            T out[K];
            for (int y = 0; y < K; ++y)
            {
                const P4<R> ps = l.plane[(size_t)y * N + s];
                T vs[6];
                for (int i = 0; i < 6; ++i)
                    vs[i] = std::fma((T)ps.x, X[i], std::fma((T)ps.y, Y[i], (T)ps.z));
                T acc = 0, mn = (T)FLT_MAX;
                for (int p = 0; p < 2 * P; ++p)
                {
                    if (p == P)
                    {
                        acc += mn;
                        mn = (T)FLT_MAX;
                    }
                    T phi = 0;
                    for (int i = 0; i < 6; ++i)
                    {
                        T term = std::fabs(vs[i] - vt[p][i]);
                        phi = i == 0 ? term : phi + term;
                    }
                    phi = std::fmin(phi * rq, (T)tau_smooth);
                    T mm = std::fma(c0, phi, m_in[(size_t)p * E + e]);
                    if (mm < mn)
                        mn = mm;
                }
                acc += mn;
                out[y] = acc;
            }
            if (min_norm)
            {
                // FP16 storage: minus the message's minimum (rounded to FP16)
                T mn = out[0];
                for (int k = 1; k < K; ++k)
                    if (out[k] < mn)
                        mn = out[k];
                for (int k = 0; k < K; ++k)
                    m_out[(size_t)k * E + e] =
                        fp16_store ? (T)(float)(_Float16)(float)(out[k] - mn) : out[k] - mn;
            }
            else
            {
                T mean = 0;
                for (int k = 0; k < K; ++k)
                    mean += out[k];
                mean /= (T)K;
                for (int k = 0; k < K; ++k)
                    m_out[(size_t)k * E + e] = out[k] - mean;
            }
        }
    }

    // aggregate_belief (hbp_isp.cu:1048-1058): belief = cost + out-edge
    // messages in edge order.
    template <typename T>
    void aggregate_t(const Level<R> &l, const T *cost, const T *m_t, T *belief) const
    {
        const int N = l.N, E = l.E;
        for (int n = 0; n < N; ++n)
            for (int k = 0; k < K; ++k)
            {
                T b = cost[(size_t)k * N + n];
                for (int e = l.nb_off[n]; e < l.nb_off[n + 1]; ++e)
                    b += m_t[(size_t)k * E + e];
                belief[(size_t)k * N + n] = b;
            }
    }

    // ping_pang_msg_k (hbp_isp.cu:419-429): msg[rev e] = msg_t[e].
    template <typename T>
    void ping_pong_t(const Level<R> &l, const T *m_t, T *m) const
    {
        const int E = l.E;
        for (int e = 0; e < E; ++e)
            for (int k = 0; k < K; ++k)
                m[(size_t)k * E + l.rev[e]] = m_t[(size_t)k * E + e];
    }

    // select_belief's compaction (hbp_isp.cu:452-472) of a K x N array by the
    // ranks in `order`: slots ranked < P move to the front in slot order.
    template <typename A>
    void compact_nodes(const Level<R> &l, A *v) const
    {
        const int N = l.N;
        for (int n = 0; n < N; ++n)
        {
            int nb = 0;
            for (int k = 0; k < K; ++k)
                if (order[(size_t)k * N + n] < P)
                {
                    v[(size_t)nb * N + n] = v[(size_t)k * N + n];
                    nb++;
                }
        }
    }

    // select_msg (hbp_isp.cu:474-493): each edge's messages compacted by the
    // kept slots of its target.
    template <typename T>
    void compact_msgs(const Level<R> &l, T *m) const
    {
        const int N = l.N, E = l.E;
        for (int e = 0; e < E; ++e)
        {
            int t = l.bd[2 * (size_t)e + 1];
            int nb = 0;
            for (int k = 0; k < K; ++k)
                if (order[(size_t)k * N + t] < P)
                {
                    m[(size_t)nb * E + e] = m[(size_t)k * E + e];
                    nb++;
                }
        }
    }

    // belief_propagation (hbp_isp.cu:1206-1214, kernels :273-493), and the
    // same step of the shadow with the main run's slot choices.
    void bp(Level<R> &l)
    {
        const int N = l.N, E = l.E;
        const size_t li = (size_t)level_of(l);
        passing_t<R>(l, l.belief.data(), msg.data());
        smooth_t<R>(l, msg.data(), msg_t.data(), fp16_msg, fp16_msg);
        aggregate_t<R>(l, l.cost.data(), msg_t.data(), l.belief.data());
        ping_pong_t<R>(l, msg_t.data(), msg.data());
        if (shadow)
        {
            passing_t<S>(l, sh_belief[li].data(), sh_msg.data());
            smooth_t<S>(l, sh_msg.data(), sh_msg_t.data(), fp16_msg, false);
            for (int e = 0; e < E; ++e)
            {
                double mm = (double)msg_t[e], ms = (double)sh_msg_t[e];
                for (int k = 1; k < K; ++k)
                {
                    mm = std::min(mm, (double)msg_t[(size_t)k * E + e]);
                    ms = std::min(ms, (double)sh_msg_t[(size_t)k * E + e]);
                }
                for (int k = 0; k < K; ++k)
                {
                    const double a = (double)msg_t[(size_t)k * E + e], b = (double)sh_msg_t[(size_t)k * E + e];
                    const double d = std::fabs((a - mm) - (b - ms)), r = std::fabs(a - b);
                    err_max = d > err_max ? d : err_max;
                    err_sum += d;
                    raw_max = r > raw_max ? r : raw_max;
                    raw_sum += r;
                    ref_abs_sum += b - ms;
                    ref_abs_max = b - ms > ref_abs_max ? b - ms : ref_abs_max;
                }
            }
            err_n += (long)K * E;
            aggregate_t<S>(l, sh_cost[li].data(), sh_msg_t.data(), sh_belief[li].data());
            ping_pong_t<S>(l, sh_msg_t.data(), sh_msg.data());
        }
        // get_belief_order + select_belief + select_msg
        for (int n = 0; n < N; ++n)
        {
            int ord[K] = {0};
            for (int i = 0; i < K - 1; ++i)
                for (int j = i + 1; j < K; ++j)
                {
                    if (l.belief[(size_t)j * N + n] < l.belief[(size_t)i * N + n])
                        ord[i]++;
                    else
                        ord[j]++;
                }
            for (int k = 0; k < K; ++k)
                order[(size_t)k * N + n] = ord[k];
        }
        compact_nodes(l, l.plane.data());
        compact_nodes(l, l.cost.data());
        compact_nodes(l, l.belief.data());
        compact_msgs<R>(l, msg.data());
        if (shadow)
        {
            compact_nodes(l, sh_cost[li].data());
            compact_nodes(l, sh_belief[li].data());
            compact_msgs<S>(l, sh_msg.data());
        }
    }

    void setup(const int *level_sizes, const int *clus, const float *mean, const int *bd,
               const int *bdl)
    {
        lv.resize(L);
        size_t oc = 0, ob = 0;
        const int HW = W * H;
        std::vector<int> im_clus(HW);
        for (int i = 0; i < HW; ++i)
            im_clus[i] = i;
        for (int li = 0; li < L; ++li)
        {
            Level<R> &l = lv[li];
            l.N = level_sizes[2 * li];
            l.E = level_sizes[2 * li + 1];
            l.Nh = li + 1 < L ? level_sizes[2 * (li + 1)] : 1;
            l.clus = clus + oc;
            l.mean.assign(mean + 6 * oc, mean + 6 * (oc + l.N));
            l.bd = bd + 2 * ob;
            l.bdl = bdl + ob;
            oc += l.N;
            ob += l.E;
            // pixels grouped by node in raster order (setup_D4, hbp_isp.cu:871-891)
            l.pix_off.assign(l.N + 1, 0);
            for (int i = 0; i < HW; ++i)
                l.pix_off[im_clus[i] + 1]++;
            for (int n = 0; n < l.N; ++n)
                l.pix_off[n + 1] += l.pix_off[n];
            l.pix.resize(HW);
            {
                std::vector<int> fill(l.pix_off.begin(), l.pix_off.end() - 1);
                for (int i = 0; i < HW; ++i)
                    l.pix[fill[im_clus[i]]++] = i;
            }
            // CSR by source + reverse edge (reverse_bd_id, hbp_isp.cu:1003-1019)
            l.nb_off.assign(l.N + 1, 0);
            for (int e = 0; e < l.E; ++e)
                l.nb_off[l.bd[2 * (size_t)e] + 1]++;
            for (int n = 0; n < l.N; ++n)
                l.nb_off[n + 1] += l.nb_off[n];
            l.rev.assign(l.E, 0);
            for (int e = 0; e < l.E; ++e)
            {
                int s = l.bd[2 * (size_t)e], t = l.bd[2 * (size_t)e + 1];
                for (int r = l.nb_off[t]; r < l.nb_off[t + 1]; ++r)
                    if (l.bd[2 * (size_t)r + 1] == s)
                    {
                        l.rev[e] = r;
                        break;
                    }
            }
            // sum_to_mean + compute_dist_color_pos (hbp_isp.cu:952-970, :78-126)
            for (int c = 0; c < 5; ++c)
                for (int n = 0; n < l.N; ++n)
                    l.mean[(size_t)c * l.N + n] /= l.mean[5 * (size_t)l.N + n];
            l.dc.assign(2 * (size_t)l.E, 0);
            for (int e = 0; e < l.E; ++e)
            {
                int s = l.bd[2 * (size_t)e], t = l.bd[2 * (size_t)e + 1];
                const float *m = l.mean.data();
                float col = std::fabs(m[s] - m[t]) + std::fabs(m[l.N + s] - m[l.N + t]);
                col = col + std::fabs(m[2 * (size_t)l.N + s] - m[2 * (size_t)l.N + t]);
                float dx = m[3 * (size_t)l.N + s] - m[3 * (size_t)l.N + t];
                float dy = m[4 * (size_t)l.N + s] - m[4 * (size_t)l.N + t];
                float pos = dx * dx + dy * dy;
                l.dc[e] = (R)(float)std::exp((double)(-col / 20.0f));
                l.dc[(size_t)l.E + e] = (R)std::sqrt(pos);
            }
            // children grouped by parent (sort_clus, hbp_isp.cu:985-1001)
            l.child_off.assign(l.Nh + 1, 0);
            for (int n = 0; n < l.N; ++n)
                l.child_off[l.clus[n] + 1]++;
            for (int p = 0; p < l.Nh; ++p)
                l.child_off[p + 1] += l.child_off[p];
            l.child.resize(l.N);
            {
                std::vector<int> fill(l.child_off.begin(), l.child_off.end() - 1);
                for (int n = 0; n < l.N; ++n)
                    l.child[fill[l.clus[n]]++] = n;
            }
            l.plane.assign((size_t)K * l.N, P4<R>{0, 0, 0, 0});
            l.cost.assign((size_t)K * l.N, 0);
            l.belief.assign((size_t)K * l.N, 0);
            l.pid.assign(3 * (size_t)l.N, 0);
            if (li + 1 < L)
                for (int i = 0; i < HW; ++i)
                    im_clus[i] = l.clus[im_clus[i]];
        }
        msg.assign((size_t)K * lv[0].E, 0);
        msg_t.assign((size_t)K * lv[0].E, 0);
        s_child.assign(lv[0].N, 0);
        s_nb.assign(lv[0].N, 0);
        s_ransac.assign(lv[0].N, 0);
        order.assign((size_t)K * lv[0].N, 0);
        plane_buf.assign((size_t)P * lv[0].N, P4<R>{0, 0, 0, 0});
        if (shadow)
        {
            sh_cost.resize(L);
            sh_belief.resize(L);
            for (int li = 0; li < L; ++li)
            {
                sh_cost[li].assign((size_t)K * lv[li].N, 0);
                sh_belief[li].assign((size_t)K * lv[li].N, 0);
            }
            sh_msg.assign((size_t)K * lv[0].E, 0);
            sh_msg_t.assign((size_t)K * lv[0].E, 0);
        }
    }

    bool step_done()
    {
        steps++;
        if (max_steps >= 0 && steps >= max_steps)
            stopped = true;
        return stopped;
    }

    // hbp_g (hbp_isp.cu:1283-1311) with init_bp (:930-950).
    void hbp_level(int li)
    {
        Level<R> &l = lv[li], &h = lv[li + 1];
        std::fill(msg.begin(), msg.begin() + (size_t)K * l.E, (R)0);
        for (int n = 0; n < l.N; ++n)
            for (int p = 0; p < P; ++p)
            {
                P4<R> pr = h.plane[(size_t)p * h.N + l.clus[n]];
                l.plane[(size_t)p * l.N + n] = pr;
                l.plane[(size_t)(p + P) * l.N + n] = pr;
                l.plane[(size_t)(p + 2 * P) * l.N + n] = pr;
            }
        plane_cost(l, 0);
        plane_cost(l, P);
        l.belief = l.cost;
        if (shadow)
        {
            std::fill(sh_msg.begin(), sh_msg.begin() + (size_t)K * l.E, (S)0);
            sh_belief[(size_t)li] = sh_cost[(size_t)li];
        }
        for (int n = 0; n < l.N; ++n)
        {
            s_nb[n] = (uint32_t)l.nb_off[n];
            s_ransac[n] = (uint32_t)l.pix_off[n];
        }
        for (int p = 0; p < h.N; ++p)
            s_child[p] = (uint32_t)l.child_off[p];

        const int iter_bp = 10 + 10 * li;
        float max_dz = (float)D / 2.0f * (float)li / (float)L;
        float max_dn = 1.0f * (float)li / (float)L;
        for (int i = 0; i < iter_bp && !stopped; ++i)
        {
            int iter_random = (i <= iter_bp / 4 * 3) ? 4 : 5;
            for (int it = 0;; ++it)
            {
                if (it <= 3)
                    ransac(l);
                else if (it <= 4)
                    spatial(li);
                else if (it <= iter_random && max_dz >= 0.01f)
                {
                    random_adjust(l, (R)max_dz, (R)max_dn);
                    max_dz /= 2.0f;
                    max_dn /= 2.0f;
                }
                else
                    break;
                plane_cost(l, 2 * P);
                bp(l);
                if (step_done())
                    return;
            }
        }
    }
};

template <typename R, typename S = double>
int run(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
        const int *bdl, const uint8_t *vol, const float *wta, int W, int H, int D, float alpha,
        float tau_smooth, int min_level, long max_steps, float *disp, float *plane_out,
        float *state_belief, float *state_plane, bool fp16_msg = false, const float *volf = nullptr,
        float data_tau = 25.0f, float *disp_levels = nullptr, float *plane_levels = nullptr,
        double *shadow_stats = nullptr)
{
    if (L < 1 || min_level < 0 || min_level > L - 1)
        return -1;
    Engine<R, S> eng;
    eng.shadow = shadow_stats != nullptr;
    eng.W = W;
    eng.H = H;
    eng.D = D;
    eng.L = L;
    eng.lambda = (R)alpha;
    eng.tau = (R)data_tau; // StereoCost::m_tau: 25 Census, 0.5 MC-CNN (stereo_cost.cu:421-441)
    eng.tau_smooth = (R)tau_smooth;
    eng.vol = vol;
    eng.volf = volf;
    eng.wta = wta;
    eng.max_steps = max_steps;
    eng.fp16_msg = fp16_msg;
    eng.setup(level_sizes, clus, mean, bd, bdl);
    // map_msg (hbp_isp.cu:1081-1105) of level li: first slot among 0..3
    // holding the minimum belief; per pixel d = clamp(a*x + b*y + c, 0, D-1).
    auto map_level = [&](int li, float *d_out, float *p_out) {
        const auto &l = eng.lv[li];
        std::vector<P4<R>> best(l.N);
        for (int n = 0; n < l.N; ++n)
        {
            R mn = l.belief[n];
            for (int p = 1; p < P; ++p)
                mn = std::min(mn, l.belief[(size_t)p * l.N + n]);
            int mp = 0;
            for (int p = 0; p < P; ++p)
                if (l.belief[(size_t)p * l.N + n] == mn)
                {
                    mp = p;
                    break;
                }
            best[n] = l.plane[(size_t)mp * l.N + n];
        }
        for (int k = 0; k < l.N; ++k)
            for (int j = l.pix_off[k]; j < l.pix_off[k + 1]; ++j)
            {
                int px = l.pix[j];
                const P4<R> &pl = best[k];
                R x = (R)(px % W), y = (R)(px / W);
                R d = pl.x * x + pl.y * y + pl.z;
                d = std::fmin(std::fmax(d, (R)0), (R)(D - 1));
                d_out[px] = (float)d;
                if (p_out)
                {
                    p_out[3 * (size_t)px] = (float)pl.x;
                    p_out[3 * (size_t)px + 1] = (float)pl.y;
                    p_out[3 * (size_t)px + 2] = (float)pl.z;
                }
            }
    };
    // HBP_ISP::run_ms_vis (hbp_isp.cu:1348-1383) keeps every level's map,
    // from the top level L-1 down to min_level, at index L-1-li
    const size_t HW = (size_t)W * H;
    auto keep_level = [&](int li) {
        if (disp_levels)
            map_level(li, disp_levels + (size_t)(L - 1 - li) * HW,
                      plane_levels ? plane_levels + (size_t)(L - 1 - li) * HW * 3 : nullptr);
    };
    // top level: messages and beliefs zero, planes zero (never written by the
    // reference, hbp_isp.cu:1333-1337)
    keep_level(L - 1);
    int lm = min_level;
    for (int li = L - 2; li >= min_level; --li)
    {
        eng.hbp_level(li);
        if (eng.stopped)
        {
            lm = li;
            break;
        }
        keep_level(li);
    }
    const auto &l = eng.lv[lm];
    if (state_belief)
        for (size_t i = 0; i < (size_t)K * l.N; ++i)
            state_belief[i] = (float)l.belief[i];
    if (state_plane)
        for (size_t i = 0; i < (size_t)K * l.N; ++i)
        {
            state_plane[4 * i] = (float)l.plane[i].x;
            state_plane[4 * i + 1] = (float)l.plane[i].y;
            state_plane[4 * i + 2] = (float)l.plane[i].z;
            state_plane[4 * i + 3] = (float)l.plane[i].w;
        }
    map_level(lm, disp, plane_out);
    if (shadow_stats)
    {
        const double n = eng.err_n ? (double)eng.err_n : 1.0;
        shadow_stats[0] = eng.err_max;
        shadow_stats[1] = eng.err_sum / n;
        shadow_stats[2] = eng.ref_abs_sum / n;
        shadow_stats[3] = (double)eng.err_n;
        shadow_stats[4] = eng.raw_max;
        shadow_stats[5] = eng.raw_sum / n;
        shadow_stats[6] = eng.ref_abs_max;
    }
    return (int)eng.steps;
}
} // namespace

extern "C" {

// Each value rounded to FP16 (nearest, ties to even) and back, as the FP16
// message store does; exposed so the tests can pin it against numpy.
void orc_round_fp16(const float *in, float *out, long n)
{
    for (long i = 0; i < n; ++i)
        out[i] = (float)(_Float16)in[i];
}

// HBP_ISP(ISPData, StereoData, alpha, tau_smooth).run_ms(min_level)
// (hbp_isp.hpp:288-386, hbp_isp.cu:1313-1346) on a segmentation pyramid in
// the ISP layout of orc_segment, the u8 disparity-major cost volume and the
// WTA disparity. mode 0: float, the engine's arithmetic; 1: the FP64 oracle;
// 2: float with messages stored as FP16 after subtracting each message's
// minimum (the engine's msg_fp16 path). max_steps >= 0 stops after
// that many candidate/BP steps and reports the current level's beliefs and
// planes (K x N, plane as 4 floats) in state_*; otherwise those are filled
// for min_level. Returns the number of BP steps run, or < 0 on bad input.
int orc_hbp(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
            const int *bdl, const uint8_t *vol, const float *wta, int W, int H, int D,
            float alpha, float tau_smooth, int min_level, int mode, long max_steps, float *disp,
            float *plane, float *state_belief, float *state_plane)
{
    if (mode == 2)
        return run<float>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha, tau_smooth,
                          min_level, max_steps, disp, plane, state_belief, state_plane, true);
    if (mode == 1)
        return run<double>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha,
                           tau_smooth, min_level, max_steps, disp, plane, state_belief,
                           state_plane);
    return run<float>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha, tau_smooth,
                      min_level, max_steps, disp, plane, state_belief, state_plane);
}

// Lock-step message error of the float run (mode 0: FP32 messages; 2: FP16
// storage), the engine's arithmetic, against a shadow run that takes the
// same discrete decisions (candidate planes, kept slots) and carries its own
// costs, beliefs and messages in double (shadow_fp64 = 1) or in float
// (shadow_fp64 = 0: the shadow repeats the float run, so every error is 0).
// The shadow normalises like the mode (mean for FP32, minimum for FP16) and
// stores unrounded. Over every message value of every BP step, with each
// message taken minus its own minimum in both runs: stats[0] the max and
// stats[1] the mean of |msg - msg_shadow|, stats[2] the mean and stats[6]
// the max of the shadow's values; stats[3] the count; stats[4] / [5] the max
// and mean of the raw difference (each run's stored normalisation). disp as
// orc_hbp. Returns the BP steps.
int orc_hbp_lockstep(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
                     const int *bdl, const uint8_t *vol, const float *wta, int W, int H, int D, float alpha,
                     float tau_smooth, int min_level, int mode, int shadow_fp64, float *disp, double *stats)
{
    if (!stats || (mode != 0 && mode != 2))
        return -1;
    if (shadow_fp64)
        return run<float, double>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha, tau_smooth,
                                  min_level, -1, disp, nullptr, nullptr, nullptr, mode == 2, nullptr, 25.0f,
                                  nullptr, nullptr, stats);
    return run<float, float>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha, tau_smooth,
                             min_level, -1, disp, nullptr, nullptr, nullptr, mode == 2, nullptr, 25.0f, nullptr,
                             nullptr, stats);
}

// The same on a float cost volume [D][H*W] (the MC-CNN path,
// stereo_cost.cu:436-441: StereoData copies the float volume and m_tau =
// data_tau, hbp_isp.hpp:91-105). Modes as orc_hbp.
int orc_hbp_f32(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
                const int *bdl, const float *volf, const float *wta, int W, int H, int D, float data_tau,
                float alpha, float tau_smooth, int min_level, int mode, long max_steps, float *disp,
                float *plane, float *state_belief, float *state_plane)
{
    if (!volf || !(data_tau > 0.0f))
        return -1;
    if (mode == 1)
        return run<double>(level_sizes, L, clus, mean, bd, bdl, nullptr, wta, W, H, D, alpha, tau_smooth,
                           min_level, max_steps, disp, plane, state_belief, state_plane, false, volf,
                           data_tau);
    return run<float>(level_sizes, L, clus, mean, bd, bdl, nullptr, wta, W, H, D, alpha, tau_smooth, min_level,
                      max_steps, disp, plane, state_belief, state_plane, mode == 2, volf, data_tau);
}

// HBP_ISP::run_ms_vis (hbp_isp.cu:1348-1383) without its superpixel image:
// the disparity (HW) and planes (HW x 3) of every level from the top level
// L-1 down to min_level, at index L-1-li of disp_levels / plane_levels
// (plane_levels may be null). vol (uint8) or volf (float, with data_tau)
// gives the data term. Modes as orc_hbp. Returns the number of BP steps.
int orc_hbp_levels(const int *level_sizes, int L, const int *clus, const float *mean, const int *bd,
                   const int *bdl, const uint8_t *vol, const float *volf, const float *wta, int W, int H, int D,
                   float data_tau, float alpha, float tau_smooth, int min_level, int mode, float *disp_levels,
                   float *plane_levels)
{
    if ((vol == nullptr) == (volf == nullptr) || !disp_levels || L < 1 || min_level < 0 || min_level > L - 1)
        return -1;
    std::vector<float> disp((size_t)W * H);
    if (mode == 1)
        return run<double>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha, tau_smooth, min_level, -1,
                           disp.data(), nullptr, nullptr, nullptr, false, volf, data_tau, disp_levels,
                           plane_levels);
    return run<float>(level_sizes, L, clus, mean, bd, bdl, vol, wta, W, H, D, alpha, tau_smooth, min_level, -1,
                      disp.data(), nullptr, nullptr, nullptr, mode == 2, volf, data_tau, disp_levels, plane_levels);
}

} // extern "C"
