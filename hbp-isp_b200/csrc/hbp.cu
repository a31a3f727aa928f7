// Hierarchical min-sum belief propagation over slanted-plane particles on the
// image segmentation pyramid. Reference: HBP_ISP (hbp_isp.hpp:122-442,
// hbp_isp.cu:1-1346).
//
// Per node K = 12 plane slots: 0-3 best, 4-7 prior (the parent's best), 8-11
// candidates. Coarse to fine, each level runs (10 + 10*level) outer
// iterations of {4 x RANSAC, 1 x spatial propagation, [1 x random adjust]}
// candidate steps; after each, the candidates' data cost is computed and one
// BP sweep passes, smooths, normalises and aggregates messages, then keeps
// the P best slots per node.
//
// Engine layout (node-major / edge-major, so the neighbour gathers of the BP
// kernels read contiguous slots): plane[n][12] float4, cost/belief[n][12],
// msg/msg_t[e][12]. Pixels of a node are listed in raster order (packed y<<16|x)
// and cut into chunks of 256 for the data cost.
//
// Reduction orders (the reference's float atomics / reduce_by_key have none):
// chunk sums over 32 slots x 8 deep combined by an xor butterfly, chunks of a
// node added in order; beliefs = cost + out-edge messages in edge order.
// Everything else follows the reference operation for operation; this file is
// compiled without multiply-add contraction so that each a*b+c rounds twice
// like the CPU oracle.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "engine.h"

namespace hbp
{
namespace
{
struct LevelDev
{
    int N, E, Nh, nchunks;
    const int *clus;         // N -> parent
    const uint32_t *pix;     // HW packed y<<16|x, sorted by (node, pixel)
    const int *pix_off;      // N + 1
    const int *chunk_off;    // N + 1
    const int *chunk_node;   // nchunks
    const int2 *bd;          // E
    const int *bdl;          // E
    const int *nb_off;       // N + 1
    const int *rev;          // E
    const float *dc;         // 2E: colour weight, centroid distance
    const float *mx, *my;    // N: centroid
    const uint32_t *child;   // N: this level's nodes grouped by parent
    const int *child_off;    // Nh + 1
    float4 *plane;           // N x K
    float *cost, *belief;    // N x K
    int4 *pid;               // N: RANSAC points (packed y<<16|x)
    unsigned long long *keep; // N: kept slots (count | 4-bit indices)
};

struct Common
{
    int W, H, D, Wp;
    float lambda, tau, tau_smooth;
    const uint8_t *vol; // [D][H][Wp]
    const float *wta;   // HW
};

__device__ __forceinline__ int px_x(uint32_t xy) { return (int)(xy & 0xffffu); }
__device__ __forceinline__ int px_y(uint32_t xy) { return (int)(xy >> 16); }

// read_plane_cost (hbp_isp.cu:205-227) for one pixel and one plane.
__device__ __forceinline__ float pixel_cost(const Common &c, int x, int y, float4 pl)
{
    float d_f = (pl.x * (float)x + pl.y * (float)y) + pl.z;
    int d = __float2int_rd(d_f);
    float cost;
    if (d < 0 || d >= c.D - 1)
        cost = c.tau;
    else
    {
        const size_t plane = (size_t)c.H * c.Wp, o = (size_t)y * c.Wp + x;
        float v0 = (float)c.vol[(size_t)d * plane + o];
        float v1 = (float)c.vol[(size_t)(d + 1) * plane + o];
        cost = ((float)(d + 1) - d_f) * v0 + (d_f - (float)d) * v1;
    }
    return c.lambda * cost;
}

// ---------------------------------------------------------------------------
// level setup
__global__ void iota_xy(uint32_t *key, uint32_t *val, const int *im_clus, int W, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        key[i] = (uint32_t)im_clus[i];
        val[i] = ((uint32_t)(i / W) << 16) | (uint32_t)(i % W);
    }
}

__global__ void compose_im_clus(const int *im, const int *clus, int n, int *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = clus[im[i]];
}

__global__ void iota_int(int *v, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        v[i] = i;
}

__global__ void count_keys(const int *k, int n, int *count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        atomicAdd(&count[k[i]], 1);
}

__global__ void chunk_counts(const int *pix_off, int N, int *nch)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N)
        nch[n] = (pix_off[n + 1] - pix_off[n] + PC_CHUNK - 1) / PC_CHUNK;
    if (n == N)
        nch[N] = 0;
}

__global__ void chunk_fill(const int *chunk_off, int N, int *chunk_node)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N)
        for (int c = chunk_off[n]; c < chunk_off[n + 1]; ++c)
            chunk_node[c] = n;
}

// reverse_bd_id_k (hbp_isp.cu:154-175): first edge t -> s in t's range.
__global__ void reverse_ids(const int2 *bd, const int *nb_off, int E, int *rev)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E)
        return;
    int2 st = bd[e];
    int r = 0;
    for (int k = nb_off[st.y]; k < nb_off[st.y + 1]; ++k)
        if (bd[k].y == st.x)
        {
            r = k;
            break;
        }
    rev[e] = r;
}

// sum_to_mean + compute_dist_color_pos + dist_trans (hbp_isp.cu:78-126,
// :952-970): colour weight exp(-(|dL| + |da| + |db|) / 20), computed in double
// and rounded once; centroid distance sqrt(dx^2 + dy^2).
__global__ void level_means(const float *sums, int N, float *mx, float *my, float *ml)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
        return;
    float w = sums[5 * (size_t)N + n];
    for (int c = 0; c < 3; ++c)
        ml[(size_t)c * N + n] = sums[(size_t)c * N + n] / w;
    mx[n] = sums[3 * (size_t)N + n] / w;
    my[n] = sums[4 * (size_t)N + n] / w;
}

__global__ void edge_weights(const int2 *bd, int E, int N, const float *ml, const float *mx,
                             const float *my, float *dc)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E)
        return;
    int s = bd[e].x, t = bd[e].y;
    float col = fabsf(ml[s] - ml[t]) + fabsf(ml[N + s] - ml[N + t]);
    col = col + fabsf(ml[2 * (size_t)N + s] - ml[2 * (size_t)N + t]);
    float dx = mx[s] - mx[t], dy = my[s] - my[t];
    float pos = dx * dx + dy * dy;
    dc[e] = (float)exp((double)(-col / 20.0f));
    dc[E + e] = sqrtf(pos);
}

// ---------------------------------------------------------------------------
// candidates
__device__ __forceinline__ float4 fit_plane(float Ax, float Ay, float Az, float Bx, float By, float Bz,
                                            float Cx, float Cy, float Cz)
{
    // fit_plane_from_points (hbp_isp.cu:531-548)
    float ax = Bx - Ax, ay = By - Ay, az = Bz - Az;
    float bx = Cx - Ax, by = Cy - Ay, bz = Cz - Az;
    float nx = ay * bz - az * by;
    float ny = az * bx - ax * bz;
    float nz = ax * by - ay * bx;
    nx /= nz;
    ny /= nz;
    nz /= nz;
    if (fabsf(nz - 1.f) > FLT_EPSILON)
        return make_float4(0.f, 0.f, (Az + Bz + Cz) / 3.f, 0.f);
    return make_float4(-nx, -ny, nx * Ax + ny * Ay + Az, 0.f);
}

// ransac_candidate_plane (hbp_isp.cu:592-640) with make_three_diff_id (:504-529).
__global__ void ransac_kernel(LevelDev lv, Common c, uint32_t *s_ransac)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= lv.N)
        return;
    const int cn = lv.pix_off[n + 1] - lv.pix_off[n], cp = lv.pix_off[n];
    if (cn <= 0) // every node owns a pixel; guard the modulo all the same
        return;
    uint32_t s = s_ransac[n];
    uint32_t xy[3] = {0, 0, 0};
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
        xy[0] = lv.pix[cp + p0];
        xy[1] = lv.pix[cp + p1];
        xy[2] = lv.pix[cp + p2];
        float X[3], Y[3], Z[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            int x = px_x(xy[k]), y = px_y(xy[k]);
            X[k] = (float)x;
            Y[k] = (float)y;
            Z[k] = c.wta[(size_t)y * c.W + x];
        }
        lv.plane[(size_t)n * K + p] = fit_plane(X[0], Y[0], Z[0], X[1], Y[1], Z[1], X[2], Y[2], Z[2]);
    }
    lv.pid[n] = make_int4((int)xy[0], (int)xy[1], (int)xy[2], 0);
    s_ransac[n] = s;
}

// random_candidate_plane + normalize_plane (hbp_isp.cu:495-503, :641-674).
__global__ void random_kernel(LevelDev lv, uint32_t *s_ransac, float max_dz, float max_dn)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= lv.N)
        return;
    uint32_t s = s_ransac[n];
    const float x = lv.mx[n], y = lv.my[n];
    for (int p = 2 * P; p < 3 * P; ++p)
    {
        float4 pl = lv.plane[(size_t)n * K + p];
        float z = pl.x * x + pl.y * y + pl.z;
        s = lcg(s);
        float dz = (float)s / 2147483648.0f * max_dz;
        z += dz;
        s = lcg(s);
        float dnx = (float)s / 2147483648.0f * max_dn;
        s = lcg(s);
        float dny = (float)s / 2147483648.0f * max_dn;
        s = lcg(s);
        float dnz = (float)s / 2147483648.0f * max_dn;
        float norm = sqrtf(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z);
        pl.x /= norm;
        pl.y /= norm;
        pl.z /= norm;
        pl.x += dnx;
        pl.y += dny;
        pl.z += dnz;
        float a = -pl.x / pl.z, b = -pl.y / pl.z;
        float cc = z - a * x - b * y;
        lv.plane[(size_t)n * K + p] = make_float4(a, b, cc, 0.f);
    }
    s_ransac[n] = s;
}

// select_child_plane (hbp_isp.cu:705-726): parent takes random children's
// slot-0 planes as its candidates.
__global__ void select_child_kernel(LevelDev lv, LevelDev h, uint32_t *s_child)
{
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= h.N)
        return;
    int cn = lv.child_off[id + 1] - lv.child_off[id], cp = lv.child_off[id];
    if (cn <= 0) // every parent has a child; guard the modulo all the same
        return;
    uint32_t s = s_child[id];
    for (int p = 0; p < P; ++p)
    {
        s = lcg(s);
        int ch = (int)lv.child[cp + (int)(s % (uint32_t)cn)];
        h.plane[(size_t)id * K + 2 * P + p] = lv.plane[(size_t)ch * K];
    }
    s_child[id] = s;
}

// neighbor_candidate_plane (hbp_isp.cu:676-703), on the parent level, seeded
// with the state kept per parent index.
__global__ void neighbor_kernel(LevelDev h, uint32_t *s_nb, float4 *buf)
{
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= h.N)
        return;
    int nbn = h.nb_off[id + 1] - h.nb_off[id], nbp = h.nb_off[id];
    if (nbn <= 0) // a level with two or more nodes is connected; guard anyway
    {
        for (int p = 0; p < P; ++p)
            buf[(size_t)id * P + p] = h.plane[(size_t)id * K + 2 * P + p];
        return;
    }
    uint32_t s = s_nb[id];
    for (int p = 0; p < P; ++p)
    {
        s = lcg(s);
        int t = h.bd[nbp + (int)(s % (uint32_t)nbn)].y;
        buf[(size_t)id * P + p] = h.plane[(size_t)t * K + 2 * P + p];
    }
    s_nb[id] = s;
}

__global__ void buf_to_candidates(LevelDev h, const float4 *buf)
{
    int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= h.N)
        return;
    for (int p = 0; p < P; ++p)
        h.plane[(size_t)id * K + 2 * P + p] = buf[(size_t)id * P + p];
}

// set_candidate_plane_k (hbp_isp.cu:727-741)
__global__ void set_candidate_kernel(LevelDev lv, LevelDev h)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= lv.N)
        return;
    int pc = lv.clus[n];
    for (int p = 2 * P; p < 3 * P; ++p)
        lv.plane[(size_t)n * K + p] = h.plane[(size_t)pc * K + p];
}

// ---------------------------------------------------------------------------
// data cost: one warp per chunk of 256 pixels of one node, 4 planes at once.
__global__ void __launch_bounds__(256) plane_cost_kernel(LevelDev lv, Common c, int sb, float4 *pc)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= lv.nchunks)
        return;
    const int n = lv.chunk_node[warp];
    const int start = lv.pix_off[n] + (warp - lv.chunk_off[n]) * PC_CHUNK;
    const int end = min(start + PC_CHUNK, lv.pix_off[n + 1]);
    float4 pl[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        pl[k] = lv.plane[(size_t)n * K + sb + k];
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int s = 0; s < PC_CHUNK / 32; ++s)
    {
        int idx = start + lane + 32 * s;
        if (idx < end)
        {
            uint32_t xy = lv.pix[idx];
            int x = px_x(xy), y = px_y(xy);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                acc[k] = acc[k] + pixel_cost(c, x, y, pl[k]);
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            acc[k] = acc[k] + __shfl_xor_sync(0xffffffffu, acc[k], off);
    if (lane == 0)
        pc[warp] = make_float4(acc[0], acc[1], acc[2], acc[3]);
}

__device__ __forceinline__ float4 node_cost(const LevelDev &lv, const float4 *pc, int n)
{
    int c0 = lv.chunk_off[n], c1 = lv.chunk_off[n + 1];
    float4 a = pc[c0];
    for (int c = c0 + 1; c < c1; ++c)
    {
        float4 b = pc[c];
        a.x = a.x + b.x;
        a.y = a.y + b.y;
        a.z = a.z + b.z;
        a.w = a.w + b.w;
    }
    return a;
}

__global__ void finalize_cost_kernel(LevelDev lv, const float4 *pc, int sb)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= lv.N)
        return;
    float4 a = node_cost(lv, pc, n);
    float *cst = lv.cost + (size_t)n * K + sb;
    cst[0] = a.x;
    cst[1] = a.y;
    cst[2] = a.z;
    cst[3] = a.w;
}

// ---------------------------------------------------------------------------
// BP step, part 1 (passing_msg_k + smooth_msg_k + normalize_msg_k,
// hbp_isp.cu:273-355): block = 32 edges x 12 slots of the source.
constexpr int BE = 32;
__global__ void __launch_bounds__(BE *K) bp_edge_kernel(LevelDev lv, Common c, const float *msg, float *msg_t)
{
    __shared__ float out[K][BE + 1];
    __shared__ float mean[BE];
    const int tx = threadIdx.x, y = threadIdx.y;
    const int e = blockIdx.x * BE + tx;
    const bool valid = e < lv.E;
    if (valid)
    {
        int2 st = lv.bd[e];
        int4 ps4 = lv.pid[st.x], pt4 = lv.pid[st.y];
        uint32_t pts[6] = {(uint32_t)ps4.x, (uint32_t)ps4.y, (uint32_t)ps4.z,
                           (uint32_t)pt4.x, (uint32_t)pt4.y, (uint32_t)pt4.z};
        float X[6], Y[6];
#pragma unroll
        for (int i = 0; i < 6; ++i)
        {
            X[i] = (float)px_x(pts[i]);
            Y[i] = (float)px_y(pts[i]);
        }
        float dist_color = fmaxf(lv.dc[e], 0.01f);
        float dist_pos = fmaxf(lv.dc[lv.E + e], 1.0f);
        float c0 = dist_color * (float)lv.bdl[e];
        float4 ps = lv.plane[(size_t)st.x * K + y];
        const float4 *pt_base = lv.plane + (size_t)st.y * K;
        const float *bt = lv.belief + (size_t)st.y * K;
        const float *me = msg + (size_t)e * K;
        float acc = 0.f, mn = FLT_MAX;
#pragma unroll
        for (int p = 0; p < 2 * P; ++p)
        {
            if (p == P)
            {
                acc = acc + mn;
                mn = FLT_MAX;
            }
            float4 pt = pt_base[p];
            float dx = ps.x - pt.x, dy = ps.y - pt.y, dz = ps.z - pt.z;
            float phi = fabsf(dx * X[0] + dy * Y[0] + dz);
#pragma unroll
            for (int i = 1; i < 6; ++i)
                phi = phi + fabsf(dx * X[i] + dy * Y[i] + dz);
            phi = fminf(phi / 3.0f / dist_pos, c.tau_smooth);
            float m = (bt[p] - me[p]) + c0 * phi;
            if (m < mn)
                mn = m;
        }
        acc = acc + mn;
        out[y][tx] = acc;
    }
    __syncthreads();
    if (valid && y == 0)
    {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < K; ++k)
            s = s + out[k][tx];
        mean[tx] = s / (float)K;
    }
    __syncthreads();
    if (valid)
        msg_t[(size_t)e * K + y] = out[y][tx] - mean[tx];
}

// BP step, part 2 (aggregate_belief_k, get_belief_order, select_belief,
// hbp_isp.cu:405-417, :432-472): per node, beliefs = cost + out-edge
// messages (edge order), rank the 12 slots by pairwise counting (a later slot
// loses ties), keep the slots ranked < P in slot order.
__global__ void bp_node_kernel(LevelDev lv, const float4 *pc, const float *msg_t)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= lv.N)
        return;
    float4 cn = node_cost(lv, pc, n);
    float *cst = lv.cost + (size_t)n * K;
    cst[8] = cn.x;
    cst[9] = cn.y;
    cst[10] = cn.z;
    cst[11] = cn.w;
    float b[K], cs[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        cs[k] = cst[k];
        b[k] = cs[k];
    }
    for (int e = lv.nb_off[n]; e < lv.nb_off[n + 1]; ++e)
    {
        const float *m = msg_t + (size_t)e * K;
#pragma unroll
        for (int k = 0; k < K; ++k)
            b[k] = b[k] + m[k];
    }
    int ord[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        ord[k] = 0;
#pragma unroll
    for (int i = 0; i < K - 1; ++i)
#pragma unroll
        for (int j = i + 1; j < K; ++j)
        {
            if (b[j] < b[i])
                ord[i]++;
            else
                ord[j]++;
        }
    float4 *pl = lv.plane + (size_t)n * K;
    float *bl = lv.belief + (size_t)n * K;
    float4 pls[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        pls[k] = pl[k];
    int nb = 0;
    unsigned long long keep = 0;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (ord[k] < P)
        {
            keep |= (unsigned long long)k << (4 + 4 * nb);
            nb++;
        }
    keep |= (unsigned long long)nb;
    // final slot j: j < nb ? kept[j] : j (in-place compaction of the reference)
#pragma unroll
    for (int j = 0; j < K; ++j)
    {
        int src = j < nb ? (int)((keep >> (4 + 4 * j)) & 15ull) : j;
        float4 p4 = pls[0];
        float bb = b[0], cc = cs[0];
#pragma unroll
        for (int k = 1; k < K; ++k)
            if (k == src)
            {
                p4 = pls[k];
                bb = b[k];
                cc = cs[k];
            }
        pl[j] = p4;
        bl[j] = bb;
        cst[j] = cc;
    }
    lv.keep[n] = keep;
}

// BP step, part 3 (ping_pang_msg_k + select_msg, hbp_isp.cu:419-429,
// :474-493): msg[rev(e)] receives msg_t[e] compacted by the kept slots of
// e's source (the target of rev(e)).
__global__ void bp_edge2_kernel(LevelDev lv, const float *msg_t, float *msg)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= lv.E)
        return;
    unsigned long long keep = lv.keep[lv.bd[e].x];
    int nb = (int)(keep & 15ull);
    const float *src = msg_t + (size_t)e * K;
    float v[K];
#pragma unroll
    for (int k = 0; k < K; ++k)
        v[k] = src[k];
    float *dst = msg + (size_t)lv.rev[e] * K;
#pragma unroll
    for (int j = 0; j < K; ++j)
    {
        int s = j < nb ? (int)((keep >> (4 + 4 * j)) & 15ull) : j;
        float o = v[0];
#pragma unroll
        for (int k = 1; k < K; ++k)
            if (k == s)
                o = v[k];
        dst[j] = o;
    }
}

// init_bp (hbp_isp.cu:930-950): priors from the parent's best slots, seeds
// from the CSR offsets.
__global__ void init_level_kernel(LevelDev lv, LevelDev h, uint32_t *s_nb, uint32_t *s_ransac,
                                  uint32_t *s_child)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < lv.N)
    {
        int pc = lv.clus[n];
        for (int p = 0; p < P; ++p)
        {
            float4 pr = h.plane[(size_t)pc * K + p];
            lv.plane[(size_t)n * K + p] = pr;
            lv.plane[(size_t)n * K + P + p] = pr;
            lv.plane[(size_t)n * K + 2 * P + p] = pr;
        }
        s_nb[n] = (uint32_t)lv.nb_off[n];
        s_ransac[n] = (uint32_t)lv.pix_off[n];
    }
    if (n < lv.Nh)
        s_child[n] = (uint32_t)lv.child_off[n];
}

__global__ void copy_cost_to_belief(LevelDev lv)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (long)lv.N * K)
        lv.belief[i] = lv.cost[i];
}

// map_msg (hbp_isp.cu:783-841): first slot among 0..3 with the minimum
// belief; per pixel d = clamp(a*x + b*y + c, 0, D-1) and the plane (a, b, c).
__global__ void map_kernel(LevelDev lv, Common c, float *disp, float *plane_out)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= lv.N)
        return;
    const float *bl = lv.belief + (size_t)n * K;
    float mn = bl[0];
    for (int p = 1; p < P; ++p)
        mn = fminf(mn, bl[p]);
    int mp = 0;
    for (int p = 0; p < P; ++p)
        if (bl[p] == mn)
        {
            mp = p;
            break;
        }
    float4 pl = lv.plane[(size_t)n * K + mp];
    for (int j = lv.pix_off[n]; j < lv.pix_off[n + 1]; ++j)
    {
        uint32_t xy = lv.pix[j];
        int x = px_x(xy), y = px_y(xy);
        float d = pl.x * (float)x + pl.y * (float)y + pl.z;
        d = fminf(fmaxf(d, 0.f), (float)(c.D - 1));
        size_t id = (size_t)y * c.W + x;
        disp[id] = d;
        if (plane_out)
        {
            plane_out[3 * id] = pl.x;
            plane_out[3 * id + 1] = pl.y;
            plane_out[3 * id + 2] = pl.z;
        }
    }
}

inline int blocks(long n, int t) { return ceil_div(n, t); }

int read_dev_int(const int *p, cudaStream_t st)
{
    int h;
    HBP_CUDA(cudaMemcpyAsync(&h, p, sizeof(int), cudaMemcpyDeviceToHost, st));
    HBP_CUDA(cudaStreamSynchronize(st));
    return h;
}
} // namespace

void hbp_infer(const Pyramid &pyr, const uint8_t *vol, int Wp, const float *wta, int D,
               const HbpParams &prm, float *disp, float *plane_out, Arena &a, cudaStream_t st)
{
    const int L = pyr.L, W = pyr.W, H = pyr.H, HW = W * H;
    const int m = prm.min_level;
    if (L < 1 || m < 0 || m > L - 1)
        throw StatusError{HBP_ERR_INVALID_ARG, "min_level must lie in [0, levels-1]"};
    if ((int)pyr.N.size() != L || (int)pyr.E.size() != L || (int)pyr.node_off.size() != L ||
        (int)pyr.edge_off.size() != L || (int)pyr.child_base.size() != L || (int)pyr.nb_base.size() != L)
        throw StatusError{HBP_ERR_INTERNAL, "pyramid bookkeeping inconsistent"};
    Common c{W, H, D, Wp, prm.alpha, CENSUS_TAU, prm.tau_smooth, vol, wta};

    size_t mark = a.mark();
    std::vector<LevelDev> lv(L);
    int Nmax = 0, Emax = 0, CHmax = 0;
    // pixel -> node per level, composed from level 0
    int *im = a.alloc<int>(HW), *im2 = a.alloc<int>(HW);
    uint32_t *kt = a.alloc<uint32_t>(HW), *ka = a.alloc<uint32_t>(HW), *va = a.alloc<uint32_t>(HW);
    int *cnt = a.alloc<int>(HW + 1);
    iota_int<<<blocks(HW, 256), 256, 0, st>>>(im, HW);
    note_launch();
    HBP_LAUNCH_CHECK();
    for (int l = 0; l < L; ++l)
    {
        LevelDev &d = lv[l];
        d = LevelDev{};
        d.N = pyr.N[l];
        d.E = pyr.E[l];
        d.Nh = l + 1 < L ? pyr.N[l + 1] : 1;
        d.clus = pyr.clus + pyr.node_off[l];
        d.bd = pyr.bd + pyr.edge_off[l];
        d.bdl = pyr.bdl + pyr.edge_off[l];
        d.nb_off = pyr.nb_off + pyr.nb_base[l];
        d.child = pyr.child + pyr.node_off[l];
        d.child_off = pyr.child_off + pyr.child_base[l];
        if (l >= m)
        {
            const int N = d.N, E = d.E;
            uint32_t *pix = a.alloc<uint32_t>(HW);
            int *pix_off = a.alloc<int>(N + 1);
            iota_xy<<<blocks(HW, 256), 256, 0, st>>>(kt, pix, im, W, HW);
            note_launch();
            HBP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (N + 1), st));
            count_keys<<<blocks(HW, 256), 256, 0, st>>>(im, HW, cnt);
            note_launch();
            HBP_LAUNCH_CHECK();
            int bits = 1;
            while ((1 << bits) < N)
                ++bits;
            radix_sort_pairs_u32(kt, pix, ka, va, HW, bits, a, st);
            exclusive_scan(cnt, pix_off, N + 1, nullptr, a, st);
            int *chunk_off = a.alloc<int>(N + 1);
            int *nch_total = a.alloc<int>(1);
            chunk_counts<<<blocks(N + 1, 256), 256, 0, st>>>(pix_off, N, cnt);
            note_launch();
            exclusive_scan(cnt, chunk_off, N + 1, nch_total, a, st);
            d.nchunks = read_dev_int(nch_total, st);
            int *chunk_node = a.alloc<int>(d.nchunks);
            chunk_fill<<<blocks(N, 256), 256, 0, st>>>(chunk_off, N, chunk_node);
            note_launch();
            HBP_LAUNCH_CHECK();
            int *rev = a.alloc<int>(E);
            reverse_ids<<<blocks(E, 256), 256, 0, st>>>(d.bd, d.nb_off, E, rev);
            note_launch();
            float *ml = a.alloc<float>(3 * (size_t)N), *mx = a.alloc<float>(N), *my = a.alloc<float>(N);
            level_means<<<blocks(N, 256), 256, 0, st>>>(pyr.sums + 6 * pyr.node_off[l], N, mx, my, ml);
            note_launch();
            float *dc = a.alloc<float>(2 * (size_t)E);
            edge_weights<<<blocks(E, 256), 256, 0, st>>>(d.bd, E, N, ml, mx, my, dc);
            note_launch();
            HBP_LAUNCH_CHECK();
            d.pix = pix;
            d.pix_off = pix_off;
            d.chunk_off = chunk_off;
            d.chunk_node = chunk_node;
            d.rev = rev;
            d.dc = dc;
            d.mx = mx;
            d.my = my;
            d.plane = a.alloc<float4>((size_t)N * K);
            d.cost = a.alloc<float>((size_t)N * K);
            d.belief = a.alloc<float>((size_t)N * K);
            d.pid = a.alloc<int4>(N);
            d.keep = a.alloc<unsigned long long>(N);
            HBP_CUDA(cudaMemsetAsync(d.plane, 0, sizeof(float4) * N * K, st));
            HBP_CUDA(cudaMemsetAsync(d.cost, 0, sizeof(float) * N * K, st));
            HBP_CUDA(cudaMemsetAsync(d.belief, 0, sizeof(float) * N * K, st));
            HBP_CUDA(cudaMemsetAsync(d.pid, 0, sizeof(int4) * N, st));
            Nmax = std::max(Nmax, N);
            Emax = std::max(Emax, E);
            CHmax = std::max(CHmax, d.nchunks);
        }
        if (l + 1 < L)
        {
            compose_im_clus<<<blocks(HW, 256), 256, 0, st>>>(im, d.clus, HW, im2);
            note_launch();
            HBP_LAUNCH_CHECK();
            std::swap(im, im2);
        }
    }
    float *msg = a.alloc<float>((size_t)Emax * K), *msg_t = a.alloc<float>((size_t)Emax * K);
    float4 *pc = a.alloc<float4>(CHmax);
    uint32_t *s_child = a.alloc<uint32_t>(Nmax), *s_nb = a.alloc<uint32_t>(Nmax),
             *s_ransac = a.alloc<uint32_t>(Nmax);
    float4 *buf = a.alloc<float4>((size_t)Nmax * P);

    auto cost_slots = [&](const LevelDev &d, int sb) {
        plane_cost_kernel<<<blocks((long)d.nchunks * 32, 256), 256, 0, st>>>(d, c, sb, pc);
        note_launch();
        finalize_cost_kernel<<<blocks(d.N, 128), 128, 0, st>>>(d, pc, sb);
        note_launch();
        HBP_LAUNCH_CHECK();
    };
    KernelProf *prof = prm.prof && prm.prof->on ? prm.prof : nullptr;
    auto bp_step = [&](const LevelDev &d) {
        if (prof)
            prof->mark(st);
        plane_cost_kernel<<<blocks((long)d.nchunks * 32, 256), 256, 0, st>>>(d, c, 2 * P, pc);
        note_launch();
        if (prof)
        {
            prof->mark(st);
            // compulsory bytes: per pixel its packed id (4 B) and two volume
            // bytes per candidate; per node 4 planes in and 4 costs out
            prof->bytes += (double)HW * (4 + 2 * P) + (double)d.N * P * (16 + 4);
            prof->launches++;
        }
        bp_edge_kernel<<<blocks(d.E, BE), dim3(BE, K), 0, st>>>(d, c, msg, msg_t);
        note_launch();
        bp_node_kernel<<<blocks(d.N, 128), 128, 0, st>>>(d, pc, msg_t);
        note_launch();
        bp_edge2_kernel<<<blocks(d.E, 128), 128, 0, st>>>(d, msg_t, msg);
        note_launch();
        HBP_LAUNCH_CHECK();
    };

    // top level: planes zero, messages and beliefs zero (hbp_isp.cu:1333-1337)
    for (int li = L - 2; li >= m; --li)
    {
        const LevelDev &d = lv[li], &h = lv[li + 1];
        HBP_CUDA(cudaMemsetAsync(msg, 0, sizeof(float) * (size_t)d.E * K, st));
        init_level_kernel<<<blocks(std::max(d.N, d.Nh), 128), 128, 0, st>>>(d, h, s_nb, s_ransac, s_child);
        note_launch();
        HBP_LAUNCH_CHECK();
        cost_slots(d, 0);
        cost_slots(d, P);
        copy_cost_to_belief<<<blocks((long)d.N * K, 256), 256, 0, st>>>(d);
        note_launch();
        HBP_LAUNCH_CHECK();
        const int iter_bp = 10 + 10 * li;
        float max_dz = (float)D / 2.0f * (float)li / (float)L;
        float max_dn = 1.0f * (float)li / (float)L;
        for (int i = 0; i < iter_bp; ++i)
        {
            const int iter_random = (i <= iter_bp / 4 * 3) ? 4 : 5;
            for (int it = 0;; ++it)
            {
                if (it <= 3)
                {
                    ransac_kernel<<<blocks(d.N, 128), 128, 0, st>>>(d, c, s_ransac);
                    note_launch();
                }
                else if (it <= 4)
                {
                    select_child_kernel<<<blocks(h.N, 128), 128, 0, st>>>(d, h, s_child);
                    note_launch();
                    neighbor_kernel<<<blocks(h.N, 128), 128, 0, st>>>(h, s_nb, buf);
                    note_launch();
                    buf_to_candidates<<<blocks(h.N, 128), 128, 0, st>>>(h, buf);
                    note_launch();
                    set_candidate_kernel<<<blocks(d.N, 128), 128, 0, st>>>(d, h);
                    note_launch();
                }
                else if (it <= iter_random && max_dz >= 0.01f)
                {
                    random_kernel<<<blocks(d.N, 128), 128, 0, st>>>(d, s_ransac, max_dz, max_dn);
                    note_launch();
                    max_dz /= 2.0f;
                    max_dn /= 2.0f;
                }
                else
                    break;
                HBP_LAUNCH_CHECK();
                bp_step(d);
            }
        }
    }
    const LevelDev &d = lv[m];
    map_kernel<<<blocks(d.N, 128), 128, 0, st>>>(d, c, disp, plane_out);
    note_launch();
    HBP_LAUNCH_CHECK();
    HBP_CUDA(cudaStreamSynchronize(st));
    a.rewind(mark);
}

} // namespace hbp
