// walls.cu -- wall-force reduction and wall integration (summation and
// integrateWalls, src/integration.cuh:191-295), in one launch.
//
// The launch also ends the step's Verlet bookkeeping (step_tail) when it
// runs on the step's own stream.  In the step graphs it runs on a branch
// instead, forked after the force kernel and joined before the next step's
// force kernel (the only reader of the wall rows), so that its serial tail
// overlaps the next step's contact search; the bookkeeping, which that
// search reads, is then a one-thread launch on the step's stream (k_tail).
//
// The wall-0 force of every particle is summed in the reference's exact
// order: 256-particle blocks in particle-index order reduced by a halving
// tree (integration.cuh:197-216), then the block partials added one after
// another in block order (integration.cuh:249-252).  The last block to finish
// (atomic ticket, no waiting) adds the partials and moves the walls.  Partials
// equal to +0.0 are skipped in that serial fold: the running sum starts at
// +0.0 and is never -0.0, so adding +0.0 leaves it unchanged bit for bit.
//
// Only the 256-blocks that the force kernel wrote a wall-0 force into this
// step (wf_flag) are read.  Every other block holds zeros only (+0.0, or a
// -0.0 that the reference's `temp = 0; temp += f` turns into +0.0), whose
// tree sum is +0.0: its partial is written as +0.0 without reading it.  An
// entry changes only when it is written, and a write flags its block, so a
// block that turned nonzero, changed or went back to zero is always read.
#include "sphk_internal.cuh"

namespace sphk {

constexpr int WALL_BLOCK = 256;

// Verlet epoch decision for the next step: lists stay exact while
// 4 * dmax < skin; otherwise every particle sweeps and a new epoch starts.
__device__ void step_tail(const Dev &d)
{
    const Params &P = *d.prm;
    Verlet &V = *d.vs;
    const float dmax = __uint_as_float(V.dmax_bits);
    const bool restart = P.skin > 0.0 && 4.0 * (double)dmax >= 0.999 * P.skin;
    V.all_rebuild = restart ? 1u : 0u;
    if (restart) V.dmax_bits = 0u;
    V.step += 1u;
}

constexpr int REF_BLOCK = 256;               // the reference's summation block
constexpr int WARPS = WALL_BLOCK / 32;        // reference blocks per CUDA block
constexpr int FOLD = 16;                      // partials per thread in the fold

template <bool TAIL>
__global__ void __launch_bounds__(WALL_BLOCK)
k_walls(Dev d)
{
    __shared__ double nz[WALL_BLOCK * FOLD];
    __shared__ uint32_t warp_tot[WARPS];
    __shared__ int is_last;
    const Params &P = *d.prm;
    const uint32_t np = P.np;
    const unsigned int t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const uint32_t nref = (np + REF_BLOCK - 1) / REF_BLOCK;

    // One warp evaluates one reference block's halving tree in its exact
    // pairing order: lane l holds c[l + 32 m], m = 0..7; levels 128, 64 and
    // 32 pair registers of a lane, levels 16..1 pair lanes (shfl_down).
    const uint32_t rb = blockIdx.x * WARPS + warp;
    if (rb < nref && d.wf_flag[rb] == 0) {
        if (lane == 0) d.wf_partial[rb] = 0.0;
    } else if (rb < nref) {
        double c[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const uint32_t idx = rb * REF_BLOCK + lane + 32u * m;
            double temp = 0.0f;
            if (idx < np) temp += d.wf_pp[idx];
            c[m] = temp;
        }
        double a0 = c[0] + c[4], a1 = c[1] + c[5], a2 = c[2] + c[6], a3 = c[3] + c[7];
        double b0 = a0 + a2, b1 = a1 + a3;
        double e = b0 + b1;
#pragma unroll
        for (int i = 16; i != 0; i /= 2) e += __shfl_down_sync(0xffffffffu, e, i);
        if (lane == 0) {
            d.wf_partial[rb] = e;
            d.wf_flag[rb] = 0;
        }
    }
    __syncthreads();
    if (t == 0) {
        __threadfence();
        const unsigned int ticket = atomicAdd(&d.walls->done_blocks, 1u);
        is_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();

    // Serial fold of the partials in block order (integration.cuh:249-252),
    // over the nonzero ones: each round loads WALL_BLOCK * FOLD partials at
    // once, compacts the nonzero ones in order into shared memory, and one
    // thread adds them up.
    double sum = 0.0;
    for (uint32_t base = 0; base < nref; base += WALL_BLOCK * FOLD) {
        double v[FOLD];
        uint32_t cnt = 0;
#pragma unroll
        for (int q = 0; q < FOLD; ++q) {
            const uint32_t b = base + t * FOLD + q;
            v[q] = (b < nref) ? __ldcg(&d.wf_partial[b]) : 0.0;
            cnt += (__double_as_longlong(v[q]) != 0ll) ? 1u : 0u;
        }
        uint32_t inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (unsigned)o) inc += y;
        }
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        uint32_t off = 0, tot = 0;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) {
            if ((unsigned)w < warp) off += warp_tot[w];
            tot += warp_tot[w];
        }
        off += inc - cnt;
#pragma unroll
        for (int q = 0; q < FOLD; ++q)
            if (__double_as_longlong(v[q]) != 0ll) nz[off++] = v[q];
        __syncthreads();
        if (t == 0)
            for (uint32_t k = 0; k < tot; ++k) sum += nz[k];
        __syncthreads();
    }

    Walls &W = *d.walls;
    const double fsum = __shfl_sync(0xffffffffu, sum, 0);   // lane 0 of warp 0 holds it
    if (t < P.nw) {
        const unsigned int w = t;
        const int wmode = P.wmode[w];
        if (wmode != 0) {
            double4 nx = W.nx[w], mvfd = W.mvfd[w];
            double vel0 = W.vel0[w];
            mvfd.z = 0.0;
            mvfd.z += fsum;
            const double dt = P.dt;
            const double sigma_0 =
                mvfd.w + P.devs_A * sin(2.0 * 3.141596654 * P.devs_f * W.t_current);
            const double N = -sigma_0 * P.L[0] * P.L[1];
            double acc = (mvfd.z + N) / mvfd.x;
            if (wmode == 2) acc = 0.0;
            vel0 += acc * dt;
            nx.w += vel0 * dt;
            mvfd.y = vel0 + 0.5 * acc * dt;
            W.nx[w] = nx;
            W.mvfd[w] = mvfd;
            W.vel0[w] = vel0;
        }
    }
    __syncthreads();
    if (t == 0) {
        W.t_current += P.dt;
        W.done_blocks = 0;
        if (TAIL) step_tail(d);
    }
}

// End of a step without walls: only the Verlet epoch bookkeeping.
__global__ void k_tail(Dev d)
{
    if (threadIdx.x == 0) step_tail(d);
}

void launch_walls(const Dev &d, uint32_t np, uint32_t nw, cudaStream_t st)
{
    if (nw == 0) {
        k_tail<<<1, 32, 0, st>>>(d);
        return;
    }
    const unsigned int nref = div_up(np, REF_BLOCK);
    k_walls<true><<<div_up(nref, WARPS), WALL_BLOCK, 0, st>>>(d);
}

// The wall reduction and integration alone (nw > 0), for a graph branch.
void launch_wall_motion(const Dev &d, uint32_t np, cudaStream_t st)
{
    const unsigned int nref = div_up(np, REF_BLOCK);
    k_walls<false><<<div_up(nref, WARPS), WALL_BLOCK, 0, st>>>(d);
}

// The Verlet bookkeeping alone.
void launch_tail(const Dev &d, cudaStream_t st)
{
    k_tail<<<1, 32, 0, st>>>(d);
}

}  // namespace sphk
