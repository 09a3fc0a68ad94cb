// dem_rebuild.cuh -- the neighbour-list rebuild as one cooperative kernel.
//
// k_rebuild is launched after k_control in every time step (a cooperative
// launch: all its blocks are resident together) and returns at once unless
// k_control set the rebuild flag (the Verlet-skin test restating
// MercuryBase::hGridNeedsRebuilding, MercuryBase.cc:496-535). One launch that
// usually does nothing costs less than a graph conditional node around ten
// kernels. When the flag is set, the blocks run the steps below in turn,
// separated by grid barriers:
//
//   1 cell keys per HGrid level and counts per cell         (keys_one)
//   2 exclusive scan of the counts, one chunk of cells per block
//   3 chunk offsets (each block sums the totals before it)
//   4 counting-sort scatter                                 (scatter_one)
//   5 per-cell ordering by particle id, counters reset      (cell_sort_one)
//   6 permutation gather of the state                       (gather_one)
//   7 neighbour lists + contact-history carry-over          (build_one)
//   8 reverse index of the new lists                        (rev_one)
//
// and block 0 makes the new state buffer and lists current. This replaces
// the HGrid buckets and the InteractionHandler lookup of the reference
// (Mercury3D.cc:224-416, InteractionHandler.cc:103-174).
//
// The barrier counter only grows: each rebuild adds gridDim.x arrivals per
// barrier, so a launch finds its base as the multiple of gridDim.x *
// RB_BARRIERS below the counter's value at its start (no block can pass the
// first barrier before every block has read it). Every wait is bounded: a
// block that polls RB_POLL_LIMIT times sets DEM_ERR_TIMEOUT and returns, and
// the host resets the counter when it sees that status.
#pragma once
#include "dem_pipeline.cuh"

namespace dem {

constexpr int RB_BLOCK = 256;
constexpr int RB_BARRIERS = 7;
constexpr long long RB_POLL_LIMIT = 1ll << 24;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

struct GridBarrier {
    unsigned long long* ctr;
    unsigned long long base;
    unsigned int passed;
};

// Thread 0 of the block waits until the counter reaches target, at most
// `limit` polls; false (and DEM_ERR_TIMEOUT in *status) if it gave up.
__device__ __forceinline__ bool wait_counter(const unsigned long long* ctr, unsigned long long target,
                                             unsigned int* status, long long limit)
{
    long long polls = 0;
    while (ld_acquire_u64(ctr) < target) {
        if (++polls > limit) {
            atomicOr(status, 1u << DEM_ERR_TIMEOUT);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// All blocks of the launch meet; false if this block gave up waiting.
__device__ __forceinline__ bool grid_barrier(GridBarrier& g, Control* ctl)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ++g.passed;
        __threadfence();
        atomicAdd(g.ctr, 1ull);
        const unsigned long long target = g.base + (unsigned long long)g.passed * gridDim.x;
        ok = wait_counter(g.ctr, target, &ctl->status, RB_POLL_LIMIT) ? 1 : 0;
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Self-test of the bounded wait: every block arrives at a barrier whose
// target one block more than the grid would have to reach, so every wait
// runs out after `limit` polls, sets DEM_ERR_TIMEOUT in *status and returns.
// Its counter is its own (reset by the caller before the launch).
__global__ void __launch_bounds__(RB_BLOCK) k_barrier_expiry(unsigned long long* ctr, unsigned int* status,
                                                             long long limit)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(ctr, 1ull);
        wait_counter(ctr, (unsigned long long)gridDim.x + 1ull, status, limit);
    }
    __syncthreads();
}

// Sum of one int per thread over the block (RB_BLOCK threads).
__device__ __forceinline__ int block_sum(int v, int* warp_sums)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = v;
    __syncthreads();
    int total = 0;
#pragma unroll
    for (int w = 0; w < RB_BLOCK / 32; ++w) total += warp_sums[w];
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(RB_BLOCK, 3) k_rebuild(DevPtrs d, unsigned long long* barrier_ctr)
{
    Control* ctl = d.ctl;
    if (!ctl->rebuild) return;
    __shared__ unsigned long long base_s;
    __shared__ int warp_sums[RB_BLOCK / 32];
    const int hc = ctl->cur, lo = ctl->lbuf; // read by every block before the first barrier
    if (threadIdx.x == 0) {
        const unsigned long long per = (unsigned long long)gridDim.x * RB_BARRIERS;
        base_s = ld_acquire_u64(barrier_ctr) / per * per;
    }
    __syncthreads();
    GridBarrier g{barrier_ctr, base_s, 0u};
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;

    // 1 keys and counts
    for (int i = gt; i < d.n; i += gs) keys_one(d, i, hc);
    if (!grid_barrier(g, ctl)) return;

    // 2 exclusive scan of this block's chunk of cells
    const int chunk = (d.ncells + gridDim.x - 1) / gridDim.x;
    const int c0 = min(d.ncells, blockIdx.x * chunk), c1 = min(d.ncells, c0 + chunk);
    int carry = 0;
    for (int t0 = c0; t0 < c1; t0 += RB_BLOCK) {
        const int i = t0 + threadIdx.x;
        const int v = i < c1 ? d.cell_count[i] : 0;
        int tile_total;
        const int ex = block_exclusive_scan(v, warp_sums, tile_total);
        if (i < c1) d.cell_start[i] = carry + ex;
        carry += tile_total;
        __syncthreads(); // warp_sums is reused by the next tile
    }
    if (threadIdx.x == 0) d.block_sums[blockIdx.x] = carry;
    if (!grid_barrier(g, ctl)) return;

    // 3 offsets of the chunks
    int part = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += RB_BLOCK) part += d.block_sums[b];
    const int off = block_sum(part, warp_sums);
    for (int i = c0 + threadIdx.x; i < c1; i += RB_BLOCK) d.cell_start[i] += off;
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) d.cell_start[d.ncells] = off + carry;
    if (!grid_barrier(g, ctl)) return;

    // 4 scatter
    for (int i = gt; i < d.n; i += gs) scatter_one(d, i);
    if (!grid_barrier(g, ctl)) return;

    // 5 id order inside each cell
    for (int cell = gt; cell < d.ncells; cell += gs) cell_sort_one(d, cell, hc);
    if (!grid_barrier(g, ctl)) return;

    // 6 gather
    for (int s = gt; s < d.n; s += gs) gather_one(d, s, hc);
    if (!grid_barrier(g, ctl)) return;

    // 7 lists and history carry-over
    for (int s = gt; s < d.n; s += gs) build_one(d, s, hc, lo);
    if (!grid_barrier(g, ctl)) return;

    // 8 reverse index of the new lists
    for (int s = gt; s < d.n; s += gs) rev_one(d, s, lo ^ 1);

    if (blockIdx.x == 0 && threadIdx.x == 0) { // the gathered state and the new lists become current
        ctl->cur = hc ^ 1;
        ctl->lbuf = lo ^ 1;
        ctl->disp_acc = 0.0;
        ctl->n_rebuilds += 1;
    }
}

} // namespace dem
