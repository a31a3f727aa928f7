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
// msg/msg_t[e][12]. Each level lists its pixels sorted by node, raster order
// inside a node (packed y<<16|x); the data cost walks that list in windows of
// 256 positions, and a node's chunks are the windows it overlaps.
//
// Reduction orders (the reference's float atomics / reduce_by_key have none):
// plane costs by the segmented-scan order described at k_cost; beliefs =
// cost + out-edge messages in edge order.
// Everything else follows the reference operation for operation; this file is
// compiled without multiply-add contraction, so each a*b+c rounds twice like
// the CPU oracle except where a fused multiply-add is written out
// (__fmaf_rn: the data cost's plane evaluation and interpolation, the
// smoothness term and the message sum).
#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <memory>
#include <vector>

#include <cuda_fp16.h>

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
    const int *chunk_off;    // N + 1: first data-cost chunk of each node
    const int *pnode;        // HW: node of each list position
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
    int W, H, D, TX; // TX: volume tiles per row
    float lambda, tau, tau_smooth; // tau: the data cost outside [0, D-1)
    const uint8_t *vol; // tiled, vol_offset() (Census: uint8 costs)
    const float *volf;  // or the same layout in floats (MC-CNN); null for uint8
    const float *wta;   // HW
};

__device__ __forceinline__ int px_x(uint32_t xy) { return (int)(xy & 0xffffu); }
__device__ __forceinline__ int px_y(uint32_t xy) { return (int)(xy >> 16); }

// A byte as float without the conversion pipe: the bits 0x4B000000 | v are
// the float 2^23 + v, so subtracting 2^23 gives v exactly.
__device__ __forceinline__ float byte_to_float(uint32_t v)
{
    return __uint_as_float(0x4B000000u | v) - 8388608.0f;
}

// read_plane_cost (hbp_isp.cu:205-227) for one pixel (xf, yf = its
// coordinates as floats, base = vol_tile_base) and one plane. For d in
// [0, D-1), (float)(d + 1) == (float)d + 1 exactly.
// F32: the float volume of the MC-CNN / AD paths (c.volf), else the uint8
// Census volume (c.vol); a template parameter, so the Census loop carries no
// branch on the volume's type.
template <bool F32>
__device__ __forceinline__ float pixel_cost(const Common &c, float xf, float yf, size_t base, float4 pl)
{
    float d_f = __fmaf_rn(pl.x, xf, __fmaf_rn(pl.y, yf, pl.z));
    int d = __float2int_rd(d_f);
    float cost;
    if (d < 0 || d >= c.D - 1)
        cost = c.tau;
    else
    {
        float v0, v1;
        if constexpr (F32)
        {
            const float *pv = c.volf + base + (size_t)d * VT_BYTES;
            v0 = pv[0];
            v1 = pv[VT_BYTES];
        }
        else
        {
            const uint8_t *pv = c.vol + base + (size_t)d * VT_BYTES;
            v0 = byte_to_float(pv[0]);
            v1 = byte_to_float(pv[VT_BYTES]);
        }
        const float fd = (float)d;
        cost = __fmaf_rn((fd + 1.0f) - d_f, v0, (d_f - fd) * v1);
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

// First list position of every node from the sorted node keys (every node
// holds at least one pixel): off[key[i]] = i where a run of equal keys
// starts, off[N] = n. No atomics: at coarse levels a count by atomics put
// every pixel on a handful of counters.
__global__ void run_starts(const uint32_t *key, int n, int N, int *off)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && (i == 0 || key[i] != key[i - 1]))
        off[key[i]] = i;
    if (i == 0)
        off[N] = n;
}

// A node's data-cost chunks are the 256-position windows of the level's pixel
// list that it overlaps.
__global__ void chunk_counts(const int *pix_off, int N, int *nch)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N)
        nch[n] = ((pix_off[n + 1] - 1) / PC_CHUNK) - (pix_off[n] / PC_CHUNK) + 1;
    if (n == N)
        nch[N] = 0;
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



// ---------------------------------------------------------------------------
// Batched BP. A batch holds up to MAXV views (one view = one pyramid + cost
// volume; a pair contributes one, or two with the right view). Every kernel
// below serves one BP phase of every participating view at once: items
// (nodes, chunks, edges) of the views are laid end to end and each thread or
// warp finds its view from the prefix table of the launch's step descriptor.
//
// A BP step of the reference (generate_plane, compute_plane_cost,
// belief_propagation; hbp_isp.cu:1206-1311) runs as
//   node phase   select of the previous step (aggregate_belief_k,
//                get_belief_order, select_belief) fused with the step's RANSAC
//                or random-adjust candidates, one thread per node;
//   [spatial]    select_child, neighbor, set_candidate (one thread per parent
//                or node);
//   data cost    read_plane_cost + the per-node reduction, one group of 4..32
//                lanes per chunk;
//   edge phase   passing_msg + smooth_msg + normalize_msg, one thread per
//                edge, with the previous step's messages pulled through
//                ping_pang_msg + select_msg (msg[e] = msg_t[rev e] compacted by
//                the kept slots of e's target).
struct ViewBufs
{
    void *msgt[2]; // [E][K] ping-pong: float, or __half when fp16
    int fp16;      // messages stored as FP16 (FP32 arithmetic)
    float4 *pc[2];  // chunk partial costs ping-pong
    uint32_t *s_child, *s_nb, *s_ransac[2];
    float4 *buf; // [Nmax][P] spatial candidates
};

struct ViewDev
{
    Common c;
    const LevelDev *lv; // [L]
    ViewBufs b;
    float *disp, *plane_out;
    float *lvl_disp, *lvl_plane; // per-level maps (run_ms_vis), index L-1-li; null if not kept
    int L;
};

constexpr int MAXV = 32; // tasks per launch descriptor

enum NodeMode
{
    NODE_SELECT = 0,
    NODE_SELECT_RANSAC = 1,
    NODE_SELECT_RANDOM = 2
};


struct Task
{
    const ViewDev *vd;             // the view's record in device memory
    const LevelDev *lvl, *lvh;     // its level li and li+1 records
    int v, li;
    int first;        // first BP step of the level: no select, zero messages
    int rb, pb, mb;   // seed buffer read / cost partials written / messages written
    int mode;         // node phase: NodeMode
    float max_dz, max_dn;
};

struct StepDesc
{
    int nt;
    int pre[MAXV + 1];
    Task t[MAXV];
};

__device__ __forceinline__ int find_task(const StepDesc &d, int item)
{
    int k = 0;
    while (k + 1 < d.nt && item >= d.pre[k + 1])
        ++k;
    return k;
}

// Select of node n (aggregate_belief_k, get_belief_order, select_belief;
// hbp_isp.cu:405-417, :432-472): belief = cost + out-edge messages in edge
// order; a slot's rank counts the slots that beat it (a later slot loses
// ties); slots ranked < P move to the front in slot order, in place.
// S3 of the data-cost order: a node's chunk sums c0..c1-1 added in order;
// the loads are issued 8 at a time (the additions stay sequential).
__device__ __forceinline__ float4 sum_chunks(const float4 *pc, int c0, int c1)
{
    float4 a = pc[c0];
    int ch = c0 + 1;
    for (; ch + 8 <= c1; ch += 8)
    {
        float4 q[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
            q[j] = pc[ch + j];
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            a.x = a.x + q[j].x;
            a.y = a.y + q[j].y;
            a.z = a.z + q[j].z;
            a.w = a.w + q[j].w;
        }
    }
    for (; ch < c1; ++ch)
    {
        const float4 q = pc[ch];
        a.x = a.x + q.x;
        a.y = a.y + q.y;
        a.z = a.z + q.z;
        a.w = a.w + q.w;
    }
    return a;
}

// msg_t[e][0..11] of buffer `buf` as floats. FP16 storage holds each value
// rounded to nearest; the arithmetic on messages is FP32 either way.
__device__ __forceinline__ void load_msg(const ViewBufs &b, int buf, size_t e, float v[K])
{
    if (b.fp16)
    {
        const uint2 *h = reinterpret_cast<const uint2 *>(static_cast<const __half *>(b.msgt[buf]) + e * K);
#pragma unroll
        for (int i = 0; i < 3; ++i)
        {
            const uint2 w = h[i];
            const float2 lo = __half22float2(*reinterpret_cast<const __half2 *>(&w.x));
            const float2 hi = __half22float2(*reinterpret_cast<const __half2 *>(&w.y));
            v[4 * i] = lo.x;
            v[4 * i + 1] = lo.y;
            v[4 * i + 2] = hi.x;
            v[4 * i + 3] = hi.y;
        }
    }
    else
    {
        const float4 *m4 = reinterpret_cast<const float4 *>(static_cast<const float *>(b.msgt[buf]) + e * K);
#pragma unroll
        for (int i = 0; i < 3; ++i)
        {
            const float4 m = m4[i];
            v[4 * i] = m.x;
            v[4 * i + 1] = m.y;
            v[4 * i + 2] = m.z;
            v[4 * i + 3] = m.w;
        }
    }
}

__device__ __forceinline__ void store_msg(const ViewBufs &b, int buf, size_t e, const float v[K])
{
    if (b.fp16)
    {
        uint2 *h = reinterpret_cast<uint2 *>(static_cast<__half *>(b.msgt[buf]) + e * K);
#pragma unroll
        for (int i = 0; i < 3; ++i)
        {
            __half2 lo = __floats2half2_rn(v[4 * i], v[4 * i + 1]);
            __half2 hi = __floats2half2_rn(v[4 * i + 2], v[4 * i + 3]);
            h[i] = make_uint2(*reinterpret_cast<uint32_t *>(&lo), *reinterpret_cast<uint32_t *>(&hi));
        }
    }
    else
    {
        float4 *o = reinterpret_cast<float4 *>(static_cast<float *>(b.msgt[buf]) + e * K);
#pragma unroll
        for (int i = 0; i < 3; ++i)
            o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    }
}

// get_belief_order + select_belief (hbp_isp.cu:432-472) for node n given its
// 12 costs cs and beliefs b: a slot's rank counts the slots that beat it (a
// later slot loses ties); slots ranked < P move to the front in slot order,
// in place; keep[n] records which.
__device__ __forceinline__ void select_finish(const LevelDev &l, int n, const float cs[K], const float b[K])
{
    float *cst = l.cost + (size_t)n * K;
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
    float *bl = l.belief + (size_t)n * K;
    float4 *pl = l.plane + (size_t)n * K;
#pragma unroll
    for (int k = 0; k < K; ++k)
    {
        bl[k] = b[k];
        cst[k] = cs[k];
    }
    int nb = 0;
    unsigned long long kl = 0;
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (ord[k] < P)
        {
            if (nb != k)
            {
                pl[nb] = pl[k];
                bl[nb] = b[k];
                cst[nb] = cs[k];
            }
            kl |= (unsigned long long)k << (4 + 4 * nb);
            nb++;
        }
    l.keep[n] = kl | (unsigned long long)nb;
}
__device__ __forceinline__ void select_thread(const LevelDev &l, int n, const float4 *pc, const ViewBufs &vb,
                                              int mbuf)
{
    float cs[K], b[K];
    const float *cst = l.cost + (size_t)n * K;
#pragma unroll
    for (int k = 0; k < 2 * P; ++k)
        cs[k] = cst[k];
    {
        const float4 a = sum_chunks(pc, l.chunk_off[n], l.chunk_off[n + 1]);
        cs[8] = a.x;
        cs[9] = a.y;
        cs[10] = a.z;
        cs[11] = a.w;
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        b[k] = cs[k];
    // out-edge messages in edge order; loads issued 4 edges at a time
    const int e0 = l.nb_off[n], e1 = l.nb_off[n + 1];
    int e = e0;
    for (; e + 4 <= e1; e += 4)
    {
        float m[4][K];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            load_msg(vb, mbuf, (size_t)(e + j), m[j]);
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int k = 0; k < K; ++k)
                b[k] = b[k] + m[j][k];
    }
    for (; e < e1; ++e)
    {
        float m[K];
        load_msg(vb, mbuf, (size_t)e, m);
#pragma unroll
        for (int k = 0; k < K; ++k)
            b[k] = b[k] + m[k];
    }
    select_finish(l, n, cs, b);
}

// The same select with one warp per node, for nodes with many chunks and
// edges (the coarse levels): the lanes load 32 chunk sums or 32 edges'
// messages at a time and walk them in order through shuffles, so the sums
// are the sequential ones of select_thread, bit for bit. Lane 0 writes.
__device__ __forceinline__ void select_warp(const LevelDev &l, int n, const float4 *pc, const ViewBufs &vb,
                                            int mbuf, int lane)
{
    float cs[K], b[K];
    const float *cst = l.cost + (size_t)n * K;
#pragma unroll
    for (int k = 0; k < 2 * P; ++k)
        cs[k] = cst[k];
    const int c0 = l.chunk_off[n], c1 = l.chunk_off[n + 1];
    float4 a = pc[c0];
    for (int base = c0 + 1; base < c1; base += 32)
    {
        const int ch = base + lane;
        const float4 q = ch < c1 ? pc[ch] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int cnt = min(32, c1 - base);
        for (int j = 0; j < cnt; ++j)
        {
            a.x = a.x + __shfl_sync(0xffffffffu, q.x, j);
            a.y = a.y + __shfl_sync(0xffffffffu, q.y, j);
            a.z = a.z + __shfl_sync(0xffffffffu, q.z, j);
            a.w = a.w + __shfl_sync(0xffffffffu, q.w, j);
        }
    }
    cs[8] = a.x;
    cs[9] = a.y;
    cs[10] = a.z;
    cs[11] = a.w;
#pragma unroll
    for (int k = 0; k < K; ++k)
        b[k] = cs[k];
    const int e0 = l.nb_off[n], e1 = l.nb_off[n + 1];
    for (int base = e0; base < e1; base += 32)
    {
        const int e = base + lane;
        float m[K];
        if (e < e1)
            load_msg(vb, mbuf, (size_t)e, m);
        else
        {
#pragma unroll
            for (int k = 0; k < K; ++k)
                m[k] = 0.f;
        }
        const int cnt = min(32, e1 - base);
        for (int j = 0; j < cnt; ++j)
#pragma unroll
            for (int k = 0; k < K; ++k)
                b[k] = b[k] + __shfl_sync(0xffffffffu, m[k], j);
    }
    if (lane == 0)
        select_finish(l, n, cs, b);
}


__device__ __forceinline__ void ransac_thread(const LevelDev &l, const Common &c, int n, uint32_t s,
                                              uint32_t *s_out)
{
    // ransac_candidate_plane + make_three_diff_id + fit_plane_from_points
    // (hbp_isp.cu:504-548, :592-640)
    const int cn = l.pix_off[n + 1] - l.pix_off[n], cp = l.pix_off[n];
    if (cn <= 0)
        return;
    // all draws first, then the pixel and WTA loads of the four candidates
    // together (two memory round trips instead of eight)
    int idx[P][3];
#pragma unroll
    for (int p = 0; p < P; ++p)
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
        idx[p][0] = p0;
        idx[p][1] = p1;
        idx[p][2] = p2;
    }
    uint32_t xy[P][3];
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            xy[p][k] = l.pix[cp + idx[p][k]];
    float Z[P][3];
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            Z[p][k] = c.wta[(size_t)px_y(xy[p][k]) * c.W + px_x(xy[p][k])];
#pragma unroll
    for (int p = 0; p < P; ++p)
        l.plane[(size_t)n * K + 2 * P + p] =
            fit_plane((float)px_x(xy[p][0]), (float)px_y(xy[p][0]), Z[p][0], (float)px_x(xy[p][1]),
                      (float)px_y(xy[p][1]), Z[p][1], (float)px_x(xy[p][2]), (float)px_y(xy[p][2]), Z[p][2]);
    l.pid[n] = make_int4((int)xy[P - 1][0], (int)xy[P - 1][1], (int)xy[P - 1][2], 0);
    *s_out = s;
}

__device__ __forceinline__ void random_thread(const LevelDev &l, int n, uint32_t s, uint32_t *s_out,
                                              float max_dz, float max_dn)
{
    // random_candidate_plane + normalize_plane (hbp_isp.cu:495-503, :641-674)
    const float x = l.mx[n], y = l.my[n];
    for (int p = 2 * P; p < 3 * P; ++p)
    {
        float4 pl = l.plane[(size_t)n * K + p];
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
        l.plane[(size_t)n * K + p] = make_float4(a, b, cc, 0.f);
    }
    *s_out = s;
}

__global__ void __launch_bounds__(128) k_node(const ViewDev *__restrict__ V, StepDesc d)
{
    int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= d.pre[d.nt])
        return;
    const Task &t = d.t[find_task(d, item)];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    const int n = item - d.pre[find_task(d, item)];
    if (!t.first)
        select_thread(l, n, v.b.pc[t.pb ^ 1], v.b, t.mb ^ 1);
    if (t.mode == NODE_SELECT_RANSAC)
        ransac_thread(l, v.c, n, v.b.s_ransac[t.rb][n], &v.b.s_ransac[t.rb ^ 1][n]);
    else if (t.mode == NODE_SELECT_RANDOM)
        random_thread(l, n, v.b.s_ransac[t.rb][n], &v.b.s_ransac[t.rb ^ 1][n], t.max_dz, t.max_dn);
}

// k_node with one warp per node (the select's sums as in select_warp; lane 0
// then draws the node's candidates).
__global__ void __launch_bounds__(128) k_node_warp(const ViewDev *__restrict__ V, StepDesc d)
{
    const int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (item >= d.pre[d.nt]) // warp-uniform
        return;
    const int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    const int n = item - d.pre[ti];
    if (!t.first)
        select_warp(l, n, v.b.pc[t.pb ^ 1], v.b, t.mb ^ 1, lane);
    if (lane != 0)
        return;
    if (t.mode == NODE_SELECT_RANSAC)
        ransac_thread(l, v.c, n, v.b.s_ransac[t.rb][n], &v.b.s_ransac[t.rb ^ 1][n]);
    else if (t.mode == NODE_SELECT_RANDOM)
        random_thread(l, n, v.b.s_ransac[t.rb][n], &v.b.s_ransac[t.rb ^ 1][n], t.max_dz, t.max_dn);
}

// select_child_plane (hbp_isp.cu:705-726), one thread per parent
__global__ void __launch_bounds__(128) k_child(const ViewDev *__restrict__ V, StepDesc d)
{
    int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= d.pre[d.nt])
        return;
    int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl, &h = *t.lvh;
    int id = item - d.pre[ti];
    int cn = l.child_off[id + 1] - l.child_off[id], cp = l.child_off[id];
    if (cn <= 0)
        return;
    uint32_t s = v.b.s_child[id];
    for (int p = 0; p < P; ++p)
    {
        s = lcg(s);
        int ch = (int)l.child[cp + (int)(s % (uint32_t)cn)];
        h.plane[(size_t)id * K + 2 * P + p] = l.plane[(size_t)ch * K];
    }
    v.b.s_child[id] = s;
}

// neighbor_candidate_plane (hbp_isp.cu:676-703) on the parent level, seeded
// with the state kept per parent index
__global__ void __launch_bounds__(128) k_neighbor(const ViewDev *__restrict__ V, StepDesc d)
{
    int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= d.pre[d.nt])
        return;
    int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &h = *t.lvh;
    int id = item - d.pre[ti];
    int nbn = h.nb_off[id + 1] - h.nb_off[id], nbp = h.nb_off[id];
    if (nbn <= 0)
    {
        for (int p = 0; p < P; ++p)
            v.b.buf[(size_t)id * P + p] = h.plane[(size_t)id * K + 2 * P + p];
        return;
    }
    uint32_t s = v.b.s_nb[id];
    for (int p = 0; p < P; ++p)
    {
        s = lcg(s);
        int tt = h.bd[nbp + (int)(s % (uint32_t)nbn)].y;
        v.b.buf[(size_t)id * P + p] = h.plane[(size_t)tt * K + 2 * P + p];
    }
    v.b.s_nb[id] = s;
}

// set_candidate_plane_k (hbp_isp.cu:727-741): children take the parent's
// spatial candidates
__global__ void __launch_bounds__(128) k_set_cand(const ViewDev *__restrict__ V, StepDesc d)
{
    int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= d.pre[d.nt])
        return;
    int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    int n = item - d.pre[ti];
    int pn = l.clus[n];
    for (int p = 0; p < P; ++p)
        l.plane[(size_t)n * K + 2 * P + p] = v.b.buf[(size_t)pn * P + p];
}

// COST_INIT: priors of the parent's best slots (init_bp + copy_prior_plane,
// hbp_isp.cu:56-73, :930-950); COST_STEP: candidates in slots 8-11.
enum CostMode
{
    COST_INIT = 0,
    COST_STEP = 1
};

// Data cost of 4 planes (read_plane_cost for every pixel, hbp_isp.cu:205-227,
// and the per-node sum of compute_plane_cost, :1159-1174). One warp = one
// 256-position window of the level's pixel list (sorted by node, raster order
// inside a node). The node sum is taken in a fixed order (the reference's
// float atomics have none; the CPU oracle restates it):
//   S0 a window that one node fills: lane j sums positions j, j+32, ...,
//      j+224 in order, then an xor butterfly (offsets 16..1) over the lanes;
// any other window is walked as 8 sub-windows of 32 positions, one per lane:
//   S1 inside each 32-position sub-window the pixels of one node form a
//      segment, summed by a segmented Hillis-Steele scan: for off = 1, 2, 4,
//      8, 16, x[r] = x[r - off] + x[r] where r - off is still in the segment;
//   S2 inside the 256-window the node's S1 pieces are added in order (a carry
//      from one sub-window to the next);
//   S3 the node's 256-window sums (its chunks, pc[]) are added in chunk order
//      by the consumers (k_init_nodes, select_thread).
__device__ __forceinline__ void emit_chunk(const LevelDev &l, float4 *pc, int n, int win, float4 v)
{
    pc[l.chunk_off[n] + win - l.pix_off[n] / PC_CHUNK] = v;
}

template <bool F32>
__device__ __forceinline__ void cost_window(const StepDesc &d, int mode, int item, int lane)
{
    const int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    const Common c = v.c;
    const int HW = c.W * c.H, N = l.N;
    const int win = item - d.pre[ti];
    float4 *pc = v.b.pc[t.pb];
    // S0: a window that one node fills entirely. The window's list entries and
    // (for a step) the node's candidate planes are loaded before the test, so
    // that their latency overlaps the node-range loads.
    if ((win + 1) * PC_CHUNK <= HW)
    {
        const int q0 = win * PC_CHUNK;
        uint32_t xy[PC_CHUNK / 32];
#pragma unroll
        for (int k = 0; k < PC_CHUNK / 32; ++k)
            xy[k] = l.pix[q0 + lane + 32 * k];
        const int n0 = l.pnode[q0];
        float4 pl[4];
        if (mode != COST_INIT)
        {
#pragma unroll
            for (int p = 0; p < P; ++p)
                pl[p] = l.plane[(size_t)n0 * K + 2 * P + p];
        }
        const int b0 = l.pix_off[n0];
        if (b0 <= q0 && l.pix_off[n0 + 1] >= q0 + PC_CHUNK) // warp-uniform
        {
            if (mode == COST_INIT)
            {
                const int pn = l.clus[n0];
#pragma unroll
                for (int p = 0; p < P; ++p)
                    pl[p] = t.lvh->plane[(size_t)pn * K + p];
                if (lane == 0 && b0 == q0) // the node's first pixel
                {
                    for (int k = 0; k < K; ++k)
                        l.plane[(size_t)n0 * K + k] = pl[k % P];
                    v.b.s_nb[n0] = (uint32_t)l.nb_off[n0];
                    v.b.s_ransac[t.rb][n0] = (uint32_t)q0;
                }
            }
            float a[4];
#pragma unroll
            for (int k = 0; k < PC_CHUNK / 32; ++k)
            {
                const int x = px_x(xy[k]), y = px_y(xy[k]);
                const float xf = (float)x, yf = (float)y;
                const size_t base = vol_tile_base(x, y, c.TX, c.D);
#pragma unroll
                for (int p = 0; p < 4; ++p)
                {
                    const float cv = pixel_cost<F32>(c, xf, yf, base, pl[p]);
                    a[p] = k == 0 ? cv : a[p] + cv;
                }
            }
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
                for (int p = 0; p < 4; ++p)
                    a[p] = a[p] + __shfl_xor_sync(0xffffffffu, a[p], off);
            if (lane == 0)
                emit_chunk(l, pc, n0, win, make_float4(a[0], a[1], a[2], a[3]));
            return;
        }
    }
    const unsigned upto = 0xffffffffu >> (31 - lane); // lanes 0..lane
    int carry_n = -1;
    float4 carry = make_float4(0.f, 0.f, 0.f, 0.f);
    int qn = win * PC_CHUNK + lane;
    int n_nx = qn < HW ? l.pnode[qn] : N;
    uint32_t xy_nx = qn < HW ? l.pix[qn] : 0u;
    for (int k = 0; k < PC_CHUNK / 32; ++k)
    {
        const int q0 = win * PC_CHUNK + 32 * k;
        if (q0 >= HW) // warp-uniform
            break;
        const int q = q0 + lane;
        const int n = n_nx;
        const uint32_t xy = xy_nx;
        if (k + 1 < PC_CHUNK / 32)
        {
            qn = q + 32;
            n_nx = qn < HW ? l.pnode[qn] : N;
            xy_nx = qn < HW ? l.pix[qn] : 0u;
        }
        // segments: heads where the node changes (positions past HW form node N)
        const int prev = __shfl_up_sync(0xffffffffu, n, 1);
        const bool head = lane == 0 || prev != n;
        const unsigned heads = __ballot_sync(0xffffffffu, head);
        const int seg = 31 - __clz(heads & upto);
        const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
        // the node carried from the previous sub-window ends there unless it
        // goes on at lane 0
        const int n_first = __shfl_sync(0xffffffffu, n, 0);
        if (lane == 0 && carry_n >= 0 && carry_n < N && carry_n != n_first)
            emit_chunk(l, pc, carry_n, win, carry);
        float cc[4] = {0.f, 0.f, 0.f, 0.f};
        if (n < N)
        {
            float4 pl[4];
            if (mode == COST_INIT)
            {
                const LevelDev &h = *t.lvh;
                const int pn = l.clus[n];
#pragma unroll
                for (int p = 0; p < P; ++p)
                    pl[p] = h.plane[(size_t)pn * K + p];
                if (head && q == l.pix_off[n])
                {
                    for (int kk = 0; kk < K; ++kk)
                        l.plane[(size_t)n * K + kk] = pl[kk % P];
                    v.b.s_nb[n] = (uint32_t)l.nb_off[n];
                    v.b.s_ransac[t.rb][n] = (uint32_t)q;
                }
            }
            else
            {
#pragma unroll
                for (int p = 0; p < P; ++p)
                    pl[p] = l.plane[(size_t)n * K + 2 * P + p];
            }
            const int x = px_x(xy), y = px_y(xy);
            const float xf = (float)x, yf = (float)y;
            const size_t base = vol_tile_base(x, y, c.TX, c.D);
#pragma unroll
            for (int p = 0; p < 4; ++p)
                cc[p] = pixel_cost<F32>(c, xf, yf, base, pl[p]);
        }
        // S1
#pragma unroll
        for (int off = 1; off < 32; off <<= 1)
#pragma unroll
            for (int p = 0; p < 4; ++p)
            {
                const float u = __shfl_up_sync(0xffffffffu, cc[p], off);
                if (lane - off >= seg)
                    cc[p] = u + cc[p];
            }
        // S2
        float4 val = make_float4(cc[0], cc[1], cc[2], cc[3]);
        if (seg == 0 && n == carry_n)
        {
            val.x = carry.x + val.x;
            val.y = carry.y + val.y;
            val.z = carry.z + val.z;
            val.w = carry.w + val.w;
        }
        if (tail && lane != 31 && n < N)
            emit_chunk(l, pc, n, win, val);
        carry.x = __shfl_sync(0xffffffffu, val.x, 31);
        carry.y = __shfl_sync(0xffffffffu, val.y, 31);
        carry.z = __shfl_sync(0xffffffffu, val.z, 31);
        carry.w = __shfl_sync(0xffffffffu, val.w, 31);
        carry_n = __shfl_sync(0xffffffffu, n, 31);
    }
    if (lane == 0 && carry_n >= 0 && carry_n < N)
        emit_chunk(l, pc, carry_n, win, carry);
}

// Blocks of COST_BLOCK threads (a warp per 256-position window), at least
// COST_MIN_BLOCKS per SM: 128 x 8 holds the same 64-register budget and
// warps per SM as 256 x 4 and ends a launch with a shorter tail.
#ifndef COST_BLOCK
#define COST_BLOCK 128
#endif
#ifndef COST_MIN_BLOCKS
#define COST_MIN_BLOCKS (1024 / COST_BLOCK)
#endif
__global__ void __launch_bounds__(COST_BLOCK, COST_MIN_BLOCKS) k_cost(const ViewDev *__restrict__ V, StepDesc d, int mode)
{
    const int item = blockIdx.x * (COST_BLOCK / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (item >= d.pre[d.nt]) // warp-uniform
        return;
    if (d.t[find_task(d, item)].vd->c.volf) // uniform per view
        cost_window<true>(d, mode, item, lane);
    else
        cost_window<false>(d, mode, item, lane);
}

// init_bp, continued: costs of the prior slots, belief = cost, child seeds.
__global__ void __launch_bounds__(128) k_init_nodes(const ViewDev *__restrict__ V, StepDesc d)
{
    int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= d.pre[d.nt])
        return;
    int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    int n = item - d.pre[ti];
    if (n < l.N)
    {
        const float4 a = sum_chunks(v.b.pc[t.pb], l.chunk_off[n], l.chunk_off[n + 1]);
        float *cs = l.cost + (size_t)n * K;
        float *bl = l.belief + (size_t)n * K;
        cs[0] = cs[4] = a.x;
        cs[1] = cs[5] = a.y;
        cs[2] = cs[6] = a.z;
        cs[3] = cs[7] = a.w;
        for (int k = 0; k < K; ++k)
            bl[k] = cs[k];
    }
    if (n < l.Nh)
        v.b.s_child[n] = (uint32_t)l.child_off[n];
}

// passing_msg_k + smooth_msg_k + normalize_msg_k (hbp_isp.cu:273-355), one
// thread per edge. EDGES_MIN_BLOCKS bounds the register count (blocks of
// 128 per SM).
#ifndef EDGES_MIN_BLOCKS
#define EDGES_MIN_BLOCKS 5
#endif
__global__ void __launch_bounds__(128, EDGES_MIN_BLOCKS) k_edges(const ViewDev *__restrict__ V, StepDesc d)
{
    int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= d.pre[d.nt])
        return;
    int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    const Common &c = v.c;
    const int e = item - d.pre[ti];
    int2 st = l.bd[e];
    // the six points, lower-index node's three first (the same order for an
    // edge and its reverse)
    int4 ps4 = l.pid[min(st.x, st.y)], pt4 = l.pid[max(st.x, st.y)];
    uint32_t pts[6] = {(uint32_t)ps4.x, (uint32_t)ps4.y, (uint32_t)ps4.z,
                       (uint32_t)pt4.x, (uint32_t)pt4.y, (uint32_t)pt4.z};
    float X[6], Y[6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
    {
        X[i] = (float)px_x(pts[i]);
        Y[i] = (float)px_y(pts[i]);
    }
    float dist_color = fmaxf(l.dc[e], 0.01f);
    float dist_pos = fmaxf(l.dc[l.E + e], 1.0f);
    float c0 = dist_color * (float)l.bdl[e];
    const float *bt = l.belief + (size_t)st.y * K;
    float mp[2 * P];
    if (t.first)
    {
#pragma unroll
        for (int p = 0; p < 2 * P; ++p)
            mp[p] = bt[p] - 0.0f;
    }
    else
    {
        unsigned long long kl = l.keep[st.y];
        int cnt = (int)(kl & 15ull);
        float vv[K];
        load_msg(v.b, t.mb ^ 1, (size_t)l.rev[e], vv);
#pragma unroll
        for (int p = 0; p < 2 * P; ++p)
        {
            int sidx = p < cnt ? (int)((kl >> (4 + 4 * p)) & 15ull) : p;
            float m = vv[0];
#pragma unroll
            for (int k = 1; k < K; ++k)
                if (k == sidx)
                    m = vv[k];
            mp[p] = bt[p] - m;
        }
    }
    // min(phi / 3 / dist_pos, tau_smooth) as min(phi * rq, tau_smooth), rq =
    // (1/3) / dist_pos rounded once per edge (the oracle states the same
    // form): every label takes the same few instructions, no division and no
    // branch per label.
    const float tau = c.tau_smooth;
    const float rq = (1.0f / 3.0f) / dist_pos;
    __shared__ float s_out[K][128];
    float sum = 0.f;
    // The eight target labels' point values are held in registers (96
    // registers, 5 blocks of 128 per SM; splitting the two label groups into
    // two passes fits 7 blocks but reloads every source plane and measured 4%
    // slower); per source label the two groups' minima, msg_t =
    // (0 + min_0) + min_1 (the reference's order). phi(y, q) = sum_i |vs_y,i - vt_q,i| with
    // v = fma(a, X_i, fma(b, Y_i, c)) (the oracle states the same form).
    {
        float vt[2 * P][6];
#pragma unroll
        for (int k = 0; k < 2 * P; ++k)
        {
            const float4 tp = l.plane[(size_t)st.y * K + k];
#pragma unroll
            for (int i = 0; i < 6; ++i)
                vt[k][i] = __fmaf_rn(tp.x, X[i], __fmaf_rn(tp.y, Y[i], tp.z));
        }
#pragma unroll 1
        for (int y = 0; y < K; ++y)
        {
            const float4 ps = l.plane[(size_t)st.x * K + y];
            float phis[2 * P];
#pragma unroll
            for (int i = 0; i < 6; ++i)
            {
                const float vs = __fmaf_rn(ps.x, X[i], __fmaf_rn(ps.y, Y[i], ps.z));
#pragma unroll
                for (int k = 0; k < 2 * P; ++k)
                    phis[k] = i == 0 ? fabsf(vs - vt[k][0]) : phis[k] + fabsf(vs - vt[k][i]);
            }
            float acc = 0.f;
#pragma unroll
            for (int g = 0; g < 2; ++g)
            {
                float mn = FLT_MAX;
#pragma unroll
                for (int k = 0; k < P; ++k)
                {
                    const float m = __fmaf_rn(c0, fminf(phis[g * P + k] * rq, tau), mp[g * P + k]);
                    if (m < mn)
                        mn = m;
                }
                acc = acc + mn;
            }
            s_out[y][threadIdx.x] = acc;
            sum = sum + acc;
        }
    }
    float out[K];
#pragma unroll
    for (int y = 0; y < K; ++y)
        out[y] = s_out[y][threadIdx.x];
    // normalise: the reference subtracts the mean (normalize_msg_k); FP16
    // storage subtracts the message's minimum instead, so the stored values
    // start at 0 and keep FP16's relative precision (the beliefs of a node
    // shift by a per-message constant, which leaves their order unchanged)
    float norm;
    if (v.b.fp16)
    {
        norm = out[0];
#pragma unroll
        for (int k = 1; k < K; ++k)
            if (out[k] < norm)
                norm = out[k];
    }
    else
        norm = sum / (float)K;
#pragma unroll
    for (int k = 0; k < K; ++k)
        out[k] = out[k] - norm;
    store_msg(v.b, t.mb, (size_t)e, out);
}

// map_msg (hbp_isp.cu:783-841), one warp per node of the task's level; into
// the view's disparity/planes, or (MAP_LEVEL) into the per-level maps of
// run_ms_vis (hbp_isp.cu:1348-1383)
constexpr int MAP_LEVEL = 1;
__global__ void __launch_bounds__(128) k_map(const ViewDev *__restrict__ V, StepDesc d)
{
    const int lane = threadIdx.x & 31;
    const int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (item >= d.pre[d.nt])
        return;
    int ti = find_task(d, item);
    const Task &t = d.t[ti];
    const ViewDev &v = *t.vd;
    const LevelDev &l = *t.lvl;
    const Common &c = v.c;
    int n = item - d.pre[ti];
    const float *bl = l.belief + (size_t)n * K;
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
    float4 pl = l.plane[(size_t)n * K + mp];
    float *disp = v.disp, *plane_out = v.plane_out;
    if (t.mode == MAP_LEVEL)
    {
        const size_t off = (size_t)(v.L - 1 - t.li) * c.W * c.H;
        disp = v.lvl_disp + off;
        plane_out = v.lvl_plane ? v.lvl_plane + 3 * off : nullptr;
    }
    for (int j = l.pix_off[n] + lane; j < l.pix_off[n + 1]; j += 32)
    {
        uint32_t xy = l.pix[j];
        int x = px_x(xy), y = px_y(xy);
        float dd = pl.x * (float)x + pl.y * (float)y + pl.z;
        dd = fminf(fmaxf(dd, 0.f), (float)(c.D - 1));
        size_t id = (size_t)y * c.W + x;
        disp[id] = dd;
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

// ---------------------------------------------------------------------------
// host side
struct ViewPlan::Impl
{
    ViewDev vd;              // host copy
    ViewDev *vd_dev = nullptr; // the same record in device memory
    std::vector<LevelDev> lv;
};

ViewPlan::ViewPlan() : impl(new Impl) {}
ViewPlan::~ViewPlan() { delete impl; }

// Per-level setup of one view (HBP_ISP constructor and the first loop of
// run_ms: setup_D4, reverse_bd_id, compute_dist_color_pos, sort_clus;
// hbp_isp.cu:871-891, :952-1019), the BP buffers, and the view descriptor.
// Persistent data go to `persist`, sort/scan temporaries to `tmp`.
void hbp_prepare(const Pyramid &pyr, const CostVolume &cv, const float *wta, int D,
                 const HbpParams &prm, float *disp, float *plane_out, Arena &persist, Arena &tmp,
                 cudaStream_t st, ViewPlan &vp)
{
    if ((cv.u8 != nullptr) == (cv.f32 != nullptr) || !(cv.tau > 0.0f))
        throw StatusError{HBP_ERR_INVALID_ARG, "exactly one cost volume (uint8 or float) and tau > 0"};
    const int L = pyr.L, W = pyr.W, H = pyr.H, HW = W * H;
    const int m = prm.min_level;
    if (L < 1 || m < 0 || m > L - 1)
        throw StatusError{HBP_ERR_INVALID_ARG, "min_level must lie in [0, levels-1]"};
    if ((int)pyr.N.size() != L || (int)pyr.E.size() != L || (int)pyr.node_off.size() != L ||
        (int)pyr.edge_off.size() != L || (int)pyr.child_base.size() != L || (int)pyr.nb_base.size() != L)
        throw StatusError{HBP_ERR_INTERNAL, "pyramid bookkeeping inconsistent"};
    Common c{W, H, D, ceil_div(W, VT_W), prm.alpha, cv.tau, prm.tau_smooth, cv.u8, cv.f32, wta};
    std::vector<LevelDev> &lv = vp.impl->lv;
    lv.assign(L, LevelDev{});
    vp.L = L;
    vp.min_level = m;
    vp.D = D;
    vp.HW = HW;
    vp.levelN.assign(L, 0);
    vp.levelE.assign(L, 0);
    vp.levelC.assign(L, 0);
    int Nmax = 1, Emax = 1, CHmax = 1;
    size_t tm = tmp.mark();
    int *im = tmp.alloc<int>(HW), *im2 = tmp.alloc<int>(HW);
    uint32_t *kt = tmp.alloc<uint32_t>(HW), *ka = tmp.alloc<uint32_t>(HW), *va = tmp.alloc<uint32_t>(HW);
    int *cnt = tmp.alloc<int>(HW + 1);
    int *nch_total = tmp.alloc<int>(1);
    iota_int<<<blocks(HW, 256), 256, 0, st>>>(im, HW);
    note_launch();
    HBP_LAUNCH_CHECK();
    for (int l = 0; l < L; ++l)
    {
        LevelDev &d = lv[l];
        d.N = pyr.N[l];
        d.E = pyr.E[l];
        d.Nh = l + 1 < L ? pyr.N[l + 1] : 1;
        d.clus = pyr.clus + pyr.node_off[l];
        d.bd = pyr.bd + pyr.edge_off[l];
        d.bdl = pyr.bdl + pyr.edge_off[l];
        d.nb_off = pyr.nb_off + pyr.nb_base[l];
        d.child = pyr.child + pyr.node_off[l];
        d.child_off = pyr.child_off + pyr.child_base[l];
        vp.levelN[l] = d.N;
        vp.levelE[l] = d.E;
        if (l >= m)
        {
            const int N = d.N, E = d.E;
            uint32_t *pix = persist.alloc<uint32_t>(HW);
            int *pix_off = persist.alloc<int>(N + 1);
            iota_xy<<<blocks(HW, 256), 256, 0, st>>>(kt, pix, im, W, HW);
            note_launch();
            HBP_LAUNCH_CHECK();
            int bits = 1;
            while ((1 << bits) < N)
                ++bits;
            radix_sort_pairs_u32(kt, pix, ka, va, HW, bits, tmp, st);
            run_starts<<<blocks(HW, 256), 256, 0, st>>>(kt, HW, N, pix_off);
            note_launch();
            HBP_LAUNCH_CHECK();
            int *chunk_off = persist.alloc<int>(N + 1);
            chunk_counts<<<blocks(N + 1, 256), 256, 0, st>>>(pix_off, N, cnt);
            note_launch();
            exclusive_scan(cnt, chunk_off, N + 1, nch_total, tmp, st);
            d.nchunks = read_dev_int(nch_total, st);
            vp.levelC[l] = d.nchunks;
            int *pnode = persist.alloc<int>(HW); // the sorted keys
            HBP_CUDA(cudaMemcpyAsync(pnode, kt, sizeof(int) * HW, cudaMemcpyDeviceToDevice, st));
            HBP_LAUNCH_CHECK();
            int *rev = persist.alloc<int>(E);
            reverse_ids<<<blocks(E, 256), 256, 0, st>>>(d.bd, d.nb_off, E, rev);
            note_launch();
            float *ml = tmp.alloc<float>(3 * (size_t)N), *mx = persist.alloc<float>(N), *my = persist.alloc<float>(N);
            level_means<<<blocks(N, 256), 256, 0, st>>>(pyr.sums + 6 * pyr.node_off[l], N, mx, my, ml);
            note_launch();
            float *dc = persist.alloc<float>(2 * (size_t)E);
            edge_weights<<<blocks(E, 256), 256, 0, st>>>(d.bd, E, N, ml, mx, my, dc);
            note_launch();
            HBP_LAUNCH_CHECK();
            d.pix = pix;
            d.pix_off = pix_off;
            d.chunk_off = chunk_off;
            d.pnode = pnode;
            d.rev = rev;
            d.dc = dc;
            d.mx = mx;
            d.my = my;
            d.plane = persist.alloc<float4>((size_t)N * K);
            d.cost = persist.alloc<float>((size_t)N * K);
            d.belief = persist.alloc<float>((size_t)N * K);
            d.pid = persist.alloc<int4>(N);
            d.keep = persist.alloc<unsigned long long>(N);
            HBP_CUDA(cudaMemsetAsync(d.plane, 0, sizeof(float4) * N * K, st));
            HBP_CUDA(cudaMemsetAsync(d.cost, 0, sizeof(float) * N * K, st));
            HBP_CUDA(cudaMemsetAsync(d.belief, 0, sizeof(float) * N * K, st));
            HBP_CUDA(cudaMemsetAsync(d.pid, 0, sizeof(int4) * N, st));
            HBP_CUDA(cudaMemsetAsync(d.keep, 0, sizeof(unsigned long long) * N, st));
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
    ViewDev &vd = vp.impl->vd;
    vd.c = c;
    vd.b.fp16 = prm.msg_fp16 ? 1 : 0;
    vd.L = L;
    LevelDev *lv_dev = persist.alloc<LevelDev>(L);
    HBP_CUDA(cudaMemcpyAsync(lv_dev, lv.data(), sizeof(LevelDev) * L, cudaMemcpyHostToDevice, st));
    vd.lv = lv_dev;
    for (int k = 0; k < 2; ++k)
    {
        vd.b.msgt[k] = prm.msg_fp16 ? (void *)persist.alloc<__half>((size_t)Emax * K)
                                    : (void *)persist.alloc<float>((size_t)Emax * K);
        vd.b.pc[k] = persist.alloc<float4>(CHmax);
        vd.b.s_ransac[k] = persist.alloc<uint32_t>(Nmax);
    }
    vd.b.s_child = persist.alloc<uint32_t>(Nmax);
    vd.b.s_nb = persist.alloc<uint32_t>(Nmax);
    vd.b.buf = persist.alloc<float4>((size_t)Nmax * P);
    vd.disp = disp;
    vd.plane_out = plane_out;
    vd.lvl_disp = prm.level_disp;
    vd.lvl_plane = prm.level_disp ? prm.level_plane : nullptr;
    vp.levels = prm.level_disp != nullptr;
    vp.impl->vd_dev = persist.alloc<ViewDev>(1);
    HBP_CUDA(cudaMemcpyAsync(vp.impl->vd_dev, &vd, sizeof(ViewDev), cudaMemcpyHostToDevice, st));
    HBP_CUDA(cudaStreamSynchronize(st)); // lv and vd (host) feed the copies above
    tmp.rewind(tm);
}

namespace
{
void launch_cost(const ViewDev *V, const StepDesc &d, int mode, cudaStream_t st)
{
    k_cost<<<blocks((long)d.pre[d.nt] * 32, COST_BLOCK), COST_BLOCK, 0, st>>>(V, d, mode);
    note_launch();
}

enum Phase
{
    PH_INIT,  // level setup: priors, their costs, beliefs, seeds (init_bp)
    PH_STEP,  // one candidate step + data cost + BP sweep
    PH_FINAL, // the level's last select
    PH_MAP_LEVEL, // map_msg of level li into the per-level maps (run_ms_vis)
    PH_MAP,   // map_msg at min_level
    PH_DONE
};

// what a launch counts per task
enum Count
{
    CNT_NODES,
    CNT_WINDOWS, // 256-position windows of the pixel list
    CNT_EDGES,
    CNT_PARENTS,
    CNT_NODES_OR_PARENTS
};
} // namespace

// One view's place in HBP_ISP::run_ms (hbp_isp.cu:1313-1346): level li, outer
// iteration i, candidate step it (0-3 RANSAC, 4 spatial, 5 random adjust).
struct BpScheduler::View
{
    ViewPlan *vp;
    void *user;
    int phase = PH_INIT, li = 0, i = 0, it = 0, step = 0, rb = 0;
    float max_dz = 0, max_dn = 0;

    int iter_bp() const { return 10 + 10 * li; }
    void enter_level(int level)
    {
        li = level;
        phase = PH_INIT;
        step = 0;
        i = 0;
        it = 0;
        max_dz = (float)vp->D / 2.0f * (float)li / (float)vp->L;
        max_dn = 1.0f * (float)li / (float)vp->L;
    }
    // skip random-adjust steps that do not apply; end the level after its
    // last iteration
    void settle()
    {
        while (phase == PH_STEP)
        {
            if (i >= iter_bp())
            {
                phase = PH_FINAL;
                break;
            }
            if (it == 5 && !(i > iter_bp() / 4 * 3 && max_dz >= 0.01f))
            {
                it = 0;
                ++i;
                continue;
            }
            break;
        }
    }
    int kind() const { return it <= 3 ? 0 : it == 4 ? 1 : 2; }
};

struct BpScheduler::Impl
{
    HbpParams prm;
    cudaStream_t st;
    std::vector<View> views;
    long ticks = 0;

    Task task_of(const View &v, bool first, int pb, int mode) const
    {
        const ViewPlan &vp = *v.vp;
        const ViewDev &vd = vp.impl->vd;
        Task t{};
        t.vd = vp.impl->vd_dev;
        t.lvl = vd.lv + v.li;
        t.lvh = v.li + 1 < vp.L ? vd.lv + v.li + 1 : t.lvl;
        t.v = 0;
        t.li = v.li;
        t.first = first ? 1 : 0;
        t.rb = v.rb;
        t.pb = pb;
        t.mb = v.step & 1;
        t.mode = mode;
        t.max_dz = v.max_dz;
        t.max_dn = v.max_dn;
        return t;
    }
    static int count_of(const View &v, int what)
    {
        const ViewPlan &vp = *v.vp;
        const int n = vp.levelN[v.li], e = vp.levelE[v.li];
        const int nh = v.li + 1 < vp.L ? vp.levelN[v.li + 1] : 1;
        const int w = (vp.HW + PC_CHUNK - 1) / PC_CHUNK;
        return what == CNT_NODES ? n : what == CNT_WINDOWS ? w : what == CNT_EDGES ? e
               : what == CNT_PARENTS ? nh : std::max(n, nh);
    }
    // Launch f(desc) over the tasks in descriptors of at most MAXV tasks.
    template <typename F>
    void launch(const std::vector<const View *> &vs, const std::vector<Task> &ts, int what, F &&f)
    {
        for (size_t b = 0; b < ts.size(); b += MAXV)
        {
            StepDesc d{};
            d.nt = (int)std::min<size_t>(MAXV, ts.size() - b);
            d.pre[0] = 0;
            for (int k = 0; k < d.nt; ++k)
            {
                d.t[k] = ts[b + k];
                d.pre[k + 1] = d.pre[k] + count_of(*vs[b + k], what);
            }
            if (d.pre[d.nt] > 0)
                f(d);
        }
    }
};

BpScheduler::BpScheduler(const HbpParams &prm, cudaStream_t st) : impl(new Impl)
{
    impl->prm = prm;
    impl->st = st;
}

BpScheduler::~BpScheduler() { delete impl; }

int BpScheduler::active() const { return (int)impl->views.size(); }

void BpScheduler::add(ViewPlan *vp, void *user)
{
    View v;
    v.vp = vp;
    v.user = user;
    if (vp->L - 2 >= vp->min_level)
    {
        if (vp->levels)
        {
            v.li = vp->L - 1; // run_ms_vis maps the top level before any BP
            v.phase = PH_MAP_LEVEL;
        }
        else
            v.enter_level(vp->L - 2);
    }
    else
    {
        v.li = vp->min_level;
        v.phase = PH_MAP;
    }
    impl->views.push_back(v);
}

// One tick: every active view takes one action; one launch per kernel kind
// (per 32 views) serves all of them. Views never read one another's data, so
// a view's results do not depend on what else is in flight.
void BpScheduler::tick(std::vector<void *> &finished)
{
    Impl &I = *impl;
    const cudaStream_t st = I.st;
    KernelProf *prof = I.prm.prof && I.prm.prof->on ? I.prm.prof : nullptr;
    KernelProf *bprof = prof && prof->breakdown ? prof : nullptr;
    const long tk = I.ticks++;
    const bool sample = bprof && tk % 8 == 0;
    auto run = [&](int kind, int li, auto &&f) {
        if (!bprof)
        {
            f();
            return;
        }
        const int tag = kind * KernelProf::LEVELS + std::min(li, KernelProf::LEVELS - 1);
        bprof->count[tag]++;
        if (sample)
        {
            bprof->markb(st);
            f();
            bprof->markb(st);
            bprof->tagb.push_back(tag);
        }
        else
            f();
    };

    std::vector<const View *> vi, vn, vs, vc, vm;
    std::vector<Task> ti, tn, ts, tc, tm;
    for (const View &v : I.views)
    {
        const bool first = v.step == 0;
        const int pb = v.step & 1;
        switch (v.phase)
        {
        case PH_INIT:
            vi.push_back(&v);
            ti.push_back(I.task_of(v, true, 0, NODE_SELECT));
            break;
        case PH_STEP:
        {
            const int k = v.kind();
            const int mode = k == 0 ? NODE_SELECT_RANSAC : k == 2 ? NODE_SELECT_RANDOM : NODE_SELECT;
            vn.push_back(&v);
            tn.push_back(I.task_of(v, first, pb, mode));
            if (k == 1)
            {
                vs.push_back(&v);
                ts.push_back(I.task_of(v, first, pb, mode));
            }
            vc.push_back(&v);
            tc.push_back(I.task_of(v, first, pb, mode));
            break;
        }
        case PH_FINAL:
            vn.push_back(&v);
            tn.push_back(I.task_of(v, false, pb, NODE_SELECT));
            break;
        case PH_MAP_LEVEL:
            vm.push_back(&v);
            tm.push_back(I.task_of(v, false, pb, MAP_LEVEL));
            break;
        case PH_MAP:
            vm.push_back(&v);
            tm.push_back(I.task_of(v, false, pb, NODE_SELECT));
            if (v.vp->levels)
            {
                vm.push_back(&v);
                tm.push_back(I.task_of(v, false, pb, MAP_LEVEL));
            }
            break;
        }
    }
    // NVTX range named after the pyramid level of the tick's first view (the
    // profiling recipes select one level of a lockstep batch with it)
    char rname[32];
    std::snprintf(rname, sizeof(rname), "bp_level_%d", I.views.empty() ? -1 : I.views[0].li);
    NvtxRange tick_range(rname);
    const int lvl_i = vi.empty() ? 0 : vi[0]->li, lvl_n = vn.empty() ? 0 : vn[0]->li;
    const int lvl_c = vc.empty() ? 0 : vc[0]->li, lvl_s = vs.empty() ? 0 : vs[0]->li;
    // level setup (init_bp): prior costs into pc[0], then costs, beliefs, seeds
    I.launch(vi, ti, CNT_WINDOWS, [&](const StepDesc &d) {
        run(6, lvl_i, [&] { launch_cost(nullptr, d, COST_INIT, st); });
    });
    I.launch(vi, ti, CNT_NODES_OR_PARENTS, [&](const StepDesc &d) {
        run(7, lvl_i, [&] { k_init_nodes<<<blocks(d.pre[d.nt], 128), 128, 0, st>>>(nullptr, d); });
        note_launch();
    });
    // node phase: select of the previous step + the step's candidates
    // large nodes (16+ chunks on average): a warp per node shortens the
    // select's serial sums; otherwise a thread per node (the same arithmetic
    // either way)
    double nch = 0, nnodes = 0;
    for (const View *v : vn)
    {
        nch += v->vp->levelC[v->li];
        nnodes += v->vp->levelN[v->li];
    }
    const bool warp_nodes = nnodes > 0 && nch >= 16.0 * nnodes;
    I.launch(vn, tn, CNT_NODES, [&](const StepDesc &d) {
        if (warp_nodes)
            run(0, lvl_n, [&] { k_node_warp<<<blocks((long)d.pre[d.nt] * 32, 128), 128, 0, st>>>(nullptr, d); });
        else
            run(0, lvl_n, [&] { k_node<<<blocks(d.pre[d.nt], 128), 128, 0, st>>>(nullptr, d); });
        note_launch();
    });
    // spatial candidates
    I.launch(vs, ts, CNT_PARENTS, [&](const StepDesc &d) {
        run(1, lvl_s, [&] { k_child<<<blocks(d.pre[d.nt], 128), 128, 0, st>>>(nullptr, d); });
        note_launch();
        run(2, lvl_s, [&] { k_neighbor<<<blocks(d.pre[d.nt], 128), 128, 0, st>>>(nullptr, d); });
        note_launch();
    });
    I.launch(vs, ts, CNT_NODES, [&](const StepDesc &d) {
        run(3, lvl_s, [&] { k_set_cand<<<blocks(d.pre[d.nt], 128), 128, 0, st>>>(nullptr, d); });
        note_launch();
    });
    // data cost of the candidates, then the BP sweep
    const bool tp = prof && !vc.empty() && (tk % 16 == 0);
    I.launch(vc, tc, CNT_WINDOWS, [&](const StepDesc &d) {
        run(4, lvl_c, [&] {
            if (tp)
                prof->mark(st);
            launch_cost(nullptr, d, COST_STEP, st);
            if (tp)
                prof->mark(st);
        });
    });
    if (tp)
    {
        // compulsory bytes of the timed data-cost launches: every pixel's list
        // entry (packed position 4 B + node 4 B) and two volume bytes per
        // candidate, plus per chunk the node's 4 planes in and 4 sums out
        for (const View *v : vc)
        {
            prof->bytes += (double)v->vp->HW * (8 + 2 * P) + (double)v->vp->levelC[v->li] * (4 * 16 + 16);
            prof->pixels += (double)v->vp->HW;
        }
        prof->launches += (long)((tc.size() + MAXV - 1) / MAXV);
    }
    I.launch(vc, tc, CNT_EDGES, [&](const StepDesc &d) {
        run(5, lvl_c, [&] {
            if (tp)
                prof->edges.mark(st);
            k_edges<<<blocks(d.pre[d.nt], 128), 128, 0, st>>>(nullptr, d);
            if (tp)
                prof->edges.mark(st);
        });
        note_launch();
    });
    if (tp)
    {
        // compulsory bytes of the timed edge-message launches: per directed
        // edge its metadata (bd 8 B, bdl 4, dc 8, rev 4) and the 12 stored
        // message values read (the reverse edge's) and written; per node of
        // the level its 12 planes, 8 beliefs, RANSAC points and kept slots
        for (const View *v : vc)
        {
            const double E = v->vp->levelE[v->li], N = v->vp->levelN[v->li];
            const double bm = I.prm.msg_fp16 ? 2.0 : 4.0;
            prof->edges.bytes += E * (24.0 + 2.0 * K * bm) + N * (K * 16.0 + 2 * P * 4.0 + 16.0 + 8.0);
            prof->edges.units += E;
        }
        prof->edges.launches += (long)((tc.size() + MAXV - 1) / MAXV);
    }
    // MAP at min_level
    if (!vm.empty())
    {
        NvtxRange map_range("bp_map");
        I.launch(vm, tm, CNT_NODES, [&](const StepDesc &d) {
            run(8, vm[0]->li, [&] { k_map<<<blocks((long)d.pre[d.nt] * 32, 128), 128, 0, st>>>(nullptr, d); });
            note_launch();
        });
    }
    HBP_LAUNCH_CHECK();
    // advance every view by the action it took
    std::vector<View> keep;
    keep.reserve(I.views.size());
    for (View &v : I.views)
    {
        switch (v.phase)
        {
        case PH_INIT:
            v.phase = PH_STEP;
            v.settle();
            break;
        case PH_STEP:
        {
            const int k = v.kind();
            v.step++;
            if (k == 0 || k == 2)
                v.rb ^= 1;
            if (k == 2)
            {
                v.max_dz /= 2.0f;
                v.max_dn /= 2.0f;
            }
            if (++v.it == 6)
            {
                v.it = 0;
                ++v.i;
            }
            v.settle();
            break;
        }
        case PH_FINAL:
            if (v.li > v.vp->min_level)
            {
                if (v.vp->levels)
                    v.phase = PH_MAP_LEVEL;
                else
                    v.enter_level(v.li - 1);
            }
            else
                v.phase = PH_MAP;
            break;
        case PH_MAP_LEVEL:
            v.enter_level(v.li - 1);
            break;
        case PH_MAP:
            v.phase = PH_DONE;
            break;
        }
        if (v.phase == PH_DONE)
            finished.push_back(v.user);
        else
            keep.push_back(v);
    }
    I.views.swap(keep);
}

BpPool::BpPool(const HbpParams &prm, int streams)
{
    HbpParams quiet = prm;
    quiet.prof = nullptr; // only the first scheduler feeds the profiler
    const int S = std::max(1, std::min(streams, 64));
    try
    {
        for (int i = 0; i < S; ++i)
        {
            cudaStream_t x;
            HBP_CUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
            st_.push_back(x);
            sc_.push_back(std::make_unique<BpScheduler>(i == 0 ? prm : quiet, x));
        }
    }
    catch (...)
    {
        sc_.clear();
        for (cudaStream_t x : st_)
            cudaStreamDestroy(x);
        throw;
    }
}

BpPool::~BpPool()
{
    for (cudaStream_t x : st_)
        cudaStreamSynchronize(x);
    sc_.clear();
    for (cudaStream_t x : st_)
        cudaStreamDestroy(x);
}

int BpPool::least_loaded() const
{
    size_t bi = 0;
    for (size_t i = 1; i < sc_.size(); ++i)
        if (sc_[i]->active() < sc_[bi]->active())
            bi = i;
    return (int)bi;
}

void BpPool::add(int i, ViewPlan *vp, void *user) { sc_[(size_t)i]->add(vp, user); }

bool BpPool::active() const
{
    for (auto &x : sc_)
        if (x->active())
            return true;
    return false;
}

void BpPool::tick(std::vector<std::pair<void *, int>> &finished)
{
    std::vector<void *> fin;
    for (size_t i = 0; i < sc_.size(); ++i)
        if (sc_[i]->active())
        {
            fin.clear();
            sc_[i]->tick(fin);
            for (void *f : fin)
                finished.emplace_back(f, (int)i);
        }
}

void BpPool::sync()
{
    for (cudaStream_t x : st_)
        HBP_CUDA(cudaStreamSynchronize(x));
}

int bp_default_streams(int views) { return std::max(1, std::min(8, (views + 1) / 2)); }

// HBP_ISP::run_ms for every view (hbp_isp.cu:1313-1346), all admitted at once,
// on a BpPool (up to 8 streams, two views each, by default).
void hbp_run_views(const std::vector<ViewPlan *> &views, const HbpParams &prm, Arena &, cudaStream_t st)
{
    HBP_CUDA(cudaStreamSynchronize(st)); // the views' setup may sit on st
    const int S = prm.bp_streams > 0 ? std::min<int>(prm.bp_streams, (int)std::max<size_t>(views.size(), 1))
                                      : bp_default_streams((int)views.size());
    BpPool pool(prm, S);
    for (size_t i = 0; i < views.size(); ++i)
        pool.add((int)(i % (size_t)S), views[i], views[i]);
    std::vector<std::pair<void *, int>> fin;
    while (pool.active())
        pool.tick(fin);
    pool.sync();
}

} // namespace hbp
