// walls.cu -- wall-force reduction and wall integration (summation and
// integrateWalls, src/integration.cuh:191-295), in one launch.
//
// The wall-0 force of every particle is summed in the reference's exact
// order: 256-particle blocks in particle-index order reduced by a halving
// tree (integration.cuh:197-216), then the block partials added one after
// another in block order (integration.cuh:249-252).  The last block to finish
// (atomic ticket, no waiting) adds the partials and moves the walls.  Partials
// equal to +0.0 are skipped in that serial fold: the running sum starts at
// +0.0 and is never -0.0, so adding +0.0 leaves it unchanged bit for bit.
#include "sphk_internal.cuh"

namespace sphk {

constexpr int WALL_BLOCK = 256;

__global__ void __launch_bounds__(WALL_BLOCK)
k_walls(Dev d)
{
    __shared__ double cache[WALL_BLOCK];
    __shared__ double nz[WALL_BLOCK];
    __shared__ int is_last;
    __shared__ int n_nz;
    const Params &P = *d.prm;
    const uint32_t np = P.np;
    const unsigned int t = threadIdx.x;
    const unsigned int nblk = gridDim.x;
    unsigned int idx = t + blockIdx.x * WALL_BLOCK;
    double temp = 0.0f;
    while (idx < np) {
        temp += d.wf_pp[idx];
        idx += WALL_BLOCK * nblk;
    }
    cache[t] = temp;
    __syncthreads();
    for (unsigned int i = WALL_BLOCK / 2; i != 0; i /= 2) {
        if (t < i) cache[t] += cache[t + i];
        __syncthreads();
    }
    if (t == 0) {
        d.wf_partial[blockIdx.x] = cache[0];
        __threadfence();
        const unsigned int ticket = atomicAdd(&d.walls->done_blocks, 1u);
        is_last = (ticket == nblk - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();

    // serial fold of the partials in block order (nonzero ones only)
    double sum = 0.0;
    for (unsigned int base = 0; base < nblk; base += WALL_BLOCK) {
        const unsigned int b = base + t;
        const double v = (b < nblk) ? __ldcg(&d.wf_partial[b]) : 0.0;
        const bool keep = (b < nblk) && (__double_as_longlong(v) != 0ll);
        // order-preserving compaction of the nonzero partials of this chunk
        const unsigned int lane = t & 31u, warp = t >> 5;
        const unsigned int bal = __ballot_sync(0xffffffffu, keep);
        __shared__ unsigned int wcount[WALL_BLOCK / 32];
        if (lane == 0) wcount[warp] = __popc(bal);
        __syncthreads();
        unsigned int off = 0;
        for (unsigned int w = 0; w < warp; ++w) off += wcount[w];
        if (keep) nz[off + __popc(bal & ((1u << lane) - 1u))] = v;
        if (t == 0) {
            unsigned int tot = 0;
            for (unsigned int w = 0; w < WALL_BLOCK / 32; ++w) tot += wcount[w];
            n_nz = (int)tot;
        }
        __syncthreads();
        if (t == 0)
            for (int k = 0; k < n_nz; ++k) sum += nz[k];
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
    }
}

void launch_walls(const Dev &d, uint32_t np, uint32_t nw, cudaStream_t st)
{
    if (nw == 0) return;
    k_walls<<<div_up(np, WALL_BLOCK), WALL_BLOCK, 0, st>>>(d);
}

}  // namespace sphk
