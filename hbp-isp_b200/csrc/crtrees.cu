// CRTrees: connected components of a directed 1-NN (functional) graph.
//
// Reference: CRTrees::get_clus (CRTrees.cu:315-354) with compute_in_degree,
// check_larger_than_one, de_link_and_compute_mask, one_step_jump, re_link,
// re_link_all, one_step_jump_max (:28-187, driven by :207-312) and
// compact_clus_label (:357-403).
// The reference drives every pointer-jumping step from the host and reads a
// flag back after each; here the whole procedure is one cooperative kernel
// whose phases are separated by bounded grid barriers, so a call costs one
// launch. Each phase reads the state left by the previous one (re_link reads
// a snapshot), which is the race-free reading of the reference's kernels; the
// labels it produces are those of the reference (checked against the
// reference build on random graphs and on every pyramid level).
#include <cooperative_groups.h>

#include <mutex>

#include "engine.h"

namespace hbp
{
namespace
{
constexpr int CR_T = 256;
constexpr int MAX_ROUNDS = 48, MAX_JUMPS = 64, MAX_FLAGS = MAX_ROUNDS * (MAX_JUMPS + 2) + MAX_JUMPS + 8;

struct CrBufs
{
    int *C, *Nb, *nn, *mask, *maskc, *indeg, *old, *M, *Kb;
};

__device__ __forceinline__ bool flag_set(int *flags, int f, bool any)
{
    if (__syncthreads_or(any) && threadIdx.x == 0)
        atomicOr(&flags[f], 1);
    return true;
}

__global__ void __launch_bounds__(CR_T)
    crtrees_kernel(const int *__restrict__ nn_in, int N, CrBufs b, int *__restrict__ label, int *flags,
                   GridBarrier bar, int *err)
{
    const unsigned nblocks = gridDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    volatile int *vflags = flags;
    int *C = b.C, *Nb = b.Nb, *nn = b.nn, *mask = b.mask, *maskc = b.maskc, *indeg = b.indeg,
        *old = b.old;
    for (int i = t0; i < N; i += stride)
    {
        int v = nn_in[i];
        nn[i] = v;
        C[i] = v;
        mask[i] = 1;
        Nb[i] = 0;
    }
    if (!grid_sync(bar, nblocks))
        return;
    int ph = 0;
    for (int round = 0;; ++round)
    {
        if (round >= MAX_ROUNDS || ph + MAX_JUMPS + 2 >= MAX_FLAGS)
        {
            if (t0 == 0)
                atomicExch(err, (int)DERR_NO_CONVERGENCE);
            return;
        }
        for (int i = t0; i < N; i += stride)
            indeg[i] = 0;
        if (!grid_sync(bar, nblocks))
            return;
        for (int i = t0; i < N; i += stride)
            if (mask[i])
                atomicAdd(&indeg[C[i]], 1);
        if (!grid_sync(bar, nblocks))
            return;
        // check_larger_than_one: any active node with in-degree > 1?
        int f = ph++;
        bool any = false;
        for (int i = t0; i < N; i += stride)
            if (mask[i] && indeg[i] > 1)
                any = true;
        flag_set(flags, f, any);
        if (!grid_sync(bar, nblocks))
            return;
        if (!vflags[f])
            break;
        // de_link_and_compute_mask
        for (int i = t0; i < N; i += stride)
        {
            int m = indeg[i] > 1;
            maskc[i] = mask[i];
            mask[i] = m;
            if (m)
                C[i] = i;
        }
        if (!grid_sync(bar, nblocks))
            return;
        // pointer_jumping: odd steps write Nb from C, even steps C from Nb
        int *cur = C, *oth = Nb;
        for (int j = 0;; ++j)
        {
            if (j >= MAX_JUMPS)
            {
                if (t0 == 0)
                    atomicExch(err, (int)DERR_NO_CONVERGENCE);
                return;
            }
            int f2 = ph++;
            any = false;
            for (int i = t0; i < N; i += stride)
                if (maskc[i])
                {
                    int a = cur[i], c2 = cur[a];
                    oth[i] = c2;
                    if (!mask[a] && mask[c2])
                        any = true;
                }
            flag_set(flags, f2, any);
            if (!grid_sync(bar, nblocks))
                return;
            int *t = cur;
            cur = oth;
            oth = t;
            if (!vflags[f2])
                break;
        }
        // re_link reads the state after jumping (buffer C)
        for (int i = t0; i < N; i += stride)
            old[i] = C[i];
        if (!grid_sync(bar, nblocks))
            return;
        for (int i = t0; i < N; i += stride)
        {
            if (mask[i])
            {
                int v = nn[i];
                C[i] = mask[v] ? v : old[v];
            }
            else if (!maskc[i])
            {
                int n2 = old[i];
                if (maskc[n2])
                    C[i] = old[n2];
            }
        }
        if (!grid_sync(bar, nblocks))
            return;
        // re_link_all
        for (int i = t0; i < N; i += stride)
        {
            int v = C[i];
            if (mask[i])
                nn[i] = v;
            else if (mask[v])
                nn[i] = C[v];
        }
        if (!grid_sync(bar, nblocks))
            return;
        for (int i = t0; i < N; i += stride)
            C[i] = nn[i];
        if (!grid_sync(bar, nblocks))
            return;
    }
    // pointer_jumping_max: label = max node index along the successor chain
    for (int i = t0; i < N; i += stride)
        b.M[i] = C[i];
    if (!grid_sync(bar, nblocks))
        return;
    int *cn = C, *on = Nb, *cm = b.M, *om = b.Kb;
    for (int j = 0;; ++j)
    {
        if (j >= MAX_JUMPS || ph >= MAX_FLAGS)
        {
            if (t0 == 0)
                atomicExch(err, (int)DERR_NO_CONVERGENCE);
            return;
        }
        int f = ph++;
        bool any = false;
        for (int i = t0; i < N; i += stride)
        {
            int a = cn[i];
            int m = max(cm[i], cm[a]);
            om[i] = m;
            on[i] = cn[a];
            if (m != cm[i])
                any = true;
        }
        flag_set(flags, f, any);
        if (!grid_sync(bar, nblocks))
            return;
        int *t = cn;
        cn = on;
        on = t;
        t = cm;
        cm = om;
        om = t;
        if (!vflags[f])
            break;
    }
    for (int i = t0; i < N; i += stride)
        label[i] = cm[i];
}

// Labels are node indices; a kernel that gave up (error word set) may leave
// garbage, so both passes check the range before indexing.
__global__ void mark_used(const int *label, int N, int *used)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N)
    {
        int l = label[i];
        if (l >= 0 && l < N)
            used[l] = 1;
    }
}

__global__ void remap_labels(const int *label, const int *pos, int N, int *clus)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N)
    {
        int l = label[i];
        clus[i] = (l >= 0 && l < N) ? pos[l] : 0;
    }
}

// Grid size of the cooperative CRTrees launch on the current device: one
// block per SM at most, which leaves room for concurrent lanes (each lane may
// run its own cooperative CRTrees launch). Computed once per device; lanes on
// several host threads may ask at the same time.
int coop_blocks(int N)
{
    static std::mutex mu;
    static int max_blocks[64] = {};
    int dev;
    HBP_CUDA(cudaGetDevice(&dev));
    int mb;
    {
        std::lock_guard<std::mutex> lk(mu);
        mb = dev >= 0 && dev < 64 ? max_blocks[dev] : 0;
    }
    if (!mb)
    {
        int sms, per_sm = 0;
        HBP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        HBP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, crtrees_kernel, CR_T, 0));
        mb = sms * (per_sm > 1 ? 1 : per_sm);
        if (mb < 1)
            mb = 1;
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 64)
            max_blocks[dev] = mb;
    }
    int want = ceil_div(N, CR_T * 4);
    return want < 1 ? 1 : (want > mb ? mb : want);
}
} // namespace

void crtrees_labels(const int *nn, int N, int *clus, int *num_dev, int *err_dev, Arena &tmp,
                    cudaStream_t st)
{
    size_t m = tmp.mark();
    CrBufs b;
    b.C = tmp.alloc<int>(N);
    b.Nb = tmp.alloc<int>(N);
    b.nn = tmp.alloc<int>(N);
    b.mask = tmp.alloc<int>(N);
    b.maskc = tmp.alloc<int>(N);
    b.indeg = tmp.alloc<int>(N);
    b.old = tmp.alloc<int>(N);
    b.M = tmp.alloc<int>(N);
    b.Kb = tmp.alloc<int>(N);
    int *label = tmp.alloc<int>(N);
    int *flags = tmp.alloc<int>(MAX_FLAGS);
    unsigned int *bar = tmp.alloc<unsigned int>(2);
    HBP_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * MAX_FLAGS, st));
    HBP_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned int) * 2, st));
    GridBarrier gb{bar, err_dev};
    int nb = coop_blocks(N);
    void *args[] = {(void *)&nn, (void *)&N, (void *)&b, (void *)&label, (void *)&flags, (void *)&gb,
                    (void *)&err_dev};
    HBP_CUDA(cudaLaunchCooperativeKernel((const void *)crtrees_kernel, dim3(nb), dim3(CR_T), args, 0, st));
    note_launch();
    // compact_clus_label: rank labels in increasing order
    int *used = b.C, *pos = b.Nb; // reuse
    HBP_CUDA(cudaMemsetAsync(used, 0, sizeof(int) * N, st));
    mark_used<<<ceil_div(N, 256), 256, 0, st>>>(label, N, used);
    note_launch();
    HBP_LAUNCH_CHECK();
    exclusive_scan(used, pos, N, num_dev, tmp, st);
    remap_labels<<<ceil_div(N, 256), 256, 0, st>>>(label, pos, N, clus);
    note_launch();
    HBP_LAUNCH_CHECK();
    tmp.rewind(m);
}

// A bounded wait that nothing ends: one block waits at a grid barrier for a
// second block that is never launched; after spin_limit polls the barrier
// records DERR_BARRIER_TIMEOUT and the kernel returns (the check that a
// device wait ends with a status instead of hanging).
__global__ void barrier_probe_kernel(GridBarrier bar, long spin_limit) { grid_sync(bar, 2u, spin_limit); }

void launch_barrier_probe(unsigned int *count2, int *err, long spin_limit, cudaStream_t st)
{
    GridBarrier b{count2, err};
    barrier_probe_kernel<<<1, 32, 0, st>>>(b, spin_limit);
    note_launch();
    HBP_LAUNCH_CHECK();
}

} // namespace hbp
