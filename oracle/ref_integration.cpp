/*
 * oracle/ref_integration.cpp -- translation unit for the reference's
 * src/integration.cuh (TEST INFRASTRUCTURE ONLY; see oracle/oracle.h).
 *
 * summation() (integration.cuh:191-221) keeps its partial sums in a
 * __shared__ array shared by a 256-thread block; here __shared__ becomes
 * `static`, and ref_summation_blocks() runs each block with 256 real threads
 * and a real barrier, one block at a time, so the block-tree order of the GPU
 * build is reproduced by the reference's own code.
 */
#define REF_SHARED_STATIC 1
#define REF_CONSTANT_EXTERN 1
#include "ref_shim.h"

#include "vector_arithmetic.h"
#include "constants.cuh"
#include "integration.cuh"

#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

/* generation-counting barrier (C++17; <barrier> needs C++20, under which the
 * CUDA host headers clash with std::lerp) */
class HostBarrier {
  public:
    explicit HostBarrier(unsigned int n) : n_(n) {}
    void arrive_and_wait()
    {
        std::unique_lock<std::mutex> lk(m_);
        unsigned int gen = gen_;
        if (++count_ == n_) {
            count_ = 0;
            ++gen_;
            cv_.notify_all();
        } else {
            cv_.wait(lk, [&] { return gen != gen_; });
        }
    }

  private:
    std::mutex m_;
    std::condition_variable cv_;
    unsigned int n_, count_ = 0, gen_ = 0;
};

/* one OpenMP/host thread per particle, one-thread blocks */
void ref_integrate_one(Float4 *x_sorted, Float4 *vel_sorted, Float4 *angvel_sorted,
                       Float4 *x, Float4 *vel, Float4 *angvel, Float4 *force,
                       Float4 *torque, Float4 *angpos, Float4 *acc, Float4 *angacc,
                       Float4 *vel0, Float4 *angvel0, Float2 *xysum, unsigned int *index,
                       unsigned int i)
{
    blockIdx.x = i;
    threadIdx.x = 0;
    integrate(x_sorted, vel_sorted, angvel_sorted, x, vel, angvel, force, torque, angpos,
              acc, angacc, vel0, angvel0, xysum, index);
}

static thread_local HostBarrier *tl_block_barrier = nullptr;

void ref_block_barrier(void)
{
    if (tl_block_barrier) tl_block_barrier->arrive_and_wait();
}

/* summation<<<nblocks, 256>>>(in, out), each block on 256 host threads */
void ref_summation_blocks(Float *in, Float *out, unsigned int nblocks)
{
    const unsigned int T = 256;
    blockDim = dim3(T, 1, 1);
    gridDim = dim3(nblocks, 1, 1);
    HostBarrier block_bar(T);
    HostBarrier phase_bar(T + 1);
    volatile unsigned int cur_block = 0;
    volatile bool stop = false;
    std::vector<std::thread> pool;
    pool.reserve(T);
    for (unsigned int t = 0; t < T; ++t) {
        pool.emplace_back([&, t]() {
            tl_block_barrier = &block_bar;
            threadIdx.x = t;
            for (;;) {
                phase_bar.arrive_and_wait(); /* block start */
                if (stop) break;
                blockIdx.x = cur_block;
                summation(in, out);
                phase_bar.arrive_and_wait(); /* block done */
            }
            tl_block_barrier = nullptr;
        });
    }
    for (unsigned int b = 0; b < nblocks; ++b) {
        cur_block = b;
        phase_bar.arrive_and_wait();
        phase_bar.arrive_and_wait();
    }
    stop = true;
    phase_bar.arrive_and_wait();
    for (auto &th : pool) th.join();
    blockDim = dim3(1, 1, 1);
}

/* integrateWalls<<<1, nw>>>: each wall on its own one-thread "block" with
 * threadIdx.x == wall index */
void ref_integrate_walls(Float4 *walls_nx, Float4 *walls_mvfd, int *walls_wmode,
                         Float *partial, Float *walls_vel0, unsigned int nblocks,
                         Float t_current, unsigned int nw)
{
    blockDim = dim3(nw, 1, 1);
    gridDim = dim3(1, 1, 1);
    for (unsigned int w = 0; w < nw; ++w) {
        blockIdx.x = 0;
        threadIdx.x = w;
        integrateWalls(walls_nx, walls_mvfd, walls_wmode, partial, walls_vel0, nblocks,
                       t_current);
    }
    blockDim = dim3(1, 1, 1);
    threadIdx.x = 0;
}
