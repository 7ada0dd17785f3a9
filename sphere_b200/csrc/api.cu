// api.cu -- the C ABI of libsphk (include/sphk.h): contexts, host<->device
// transfer in the reference's host layout, and stepping through CUDA graphs.
#include "diff_step.cuh"
#include "../../include/sphk.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <map>
#include <vector>

namespace sphk {
void launch_topo(const Dev &d, uint32_t np, bool visc, int a, cudaStream_t st);
void launch_force(const Dev &d, const Params &hp, uint32_t np, int model, int a, int write_outputs,
                  cudaStream_t st);
void launch_contact(const Dev &d, const Params &hp, uint32_t np, int model, int a, int write_outputs,
                    cudaStream_t st);
void launch_bonds(const Dev &d, const Params &hp, uint32_t nb0, int a, cudaStream_t st);
void launch_bond_storage(const Dev &d, uint32_t nb0, uint32_t np, cudaStream_t st);
void launch_walls(const Dev &d, uint32_t np, uint32_t nw, cudaStream_t st);
void launch_wall_motion(const Dev &d, uint32_t np, cudaStream_t st);
void launch_tail(const Dev &d, cudaStream_t st);
void launch_cell_init(const Dev &d, uint32_t np, int a, cudaStream_t st);
void launch_epoch_reset(const Dev &d, cudaStream_t st);
void launch_rebuild(const Dev &d, uint32_t np, uint32_t ncells, int a, cudaStream_t st);
unsigned int scan_tile_count(uint32_t ncells);
void relayout(const Dev &d, uint32_t np, int a, void *scratch, cudaStream_t st);
void launch_rebuild_gate(cudaGraphConditionalHandle h, const uint32_t *rebuild, cudaStream_t st);
void launch_darcy(const Dev &d, const DarcyDev &f, const Params &hp, int a, int hs, cudaStream_t st);
struct RenderArgs;
void launch_maxpos(const Dev &d, uint32_t np, int a, unsigned long long *mx, cudaStream_t st);
int render_image(const Dev &d, uint32_t np, int a, const double L[3], const double maxpos[3],
                 const sph_render_opts &o, double *values, unsigned long long *keys, uchar4 *img,
                 float *rays, cudaStream_t st);
void launch_force_tape(const Dev &d, uint32_t np, int a, int tape_step, cudaStream_t st);
void launch_rev_step(const Dev &d, const AdjDev &a, uint32_t np, int j, cudaStream_t st);
void launch_user_to_storage3(const double *src, double4 *dst, const uint32_t *uid, uint32_t n,
                             cudaStream_t st);
void launch_user_to_storage1(const double *src, double *dst, const uint32_t *uid, double dflt,
                             uint32_t n, cudaStream_t st);
void launch_storage_to_user3(const double4 *a, const double4 *b, double *dst, const uint32_t *sidx,
                             uint32_t n, cudaStream_t st);
void launch_storage_to_user1(const double *src, double *dst, const uint32_t *sidx, uint32_t n,
                             cudaStream_t st);
}  // namespace sphk

using namespace sphk;

struct sph_ctx {
    Dev d{};
    Params hp{};                     // the first instance's parameters (all of one scene's)
    std::vector<Params> hps;         // every instance's parameters
    uint32_t np_all = 0, ncells_all = 0, ninst = 1;
    bool batched = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;     // captures the bodies of conditional graph nodes
    bool cond_rebuild = true;        // graphs skip the rebuild kernels when no cell changed
    int a = 0;                       // buffer holding the current state
    uint64_t steps = 0, relayouts = 0, since_relayout = 0;
    double t_host = 0.0;
    int64_t relayout_every = 0;
    double skin_rel = 0.1;           // Verlet skin as a fraction of the largest radius
    int graph_steps = 8;
    bool uploaded = false;
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    std::vector<void *> allocs;
    size_t device_bytes = 0;
    cudaGraphExec_t g_multi[2] = {nullptr, nullptr};
    cudaGraphExec_t g_single[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int graphs_for_k = 0;
    std::string err;
    int sticky = SPH_OK;
    // profile mode: events bracket each phase of each step
    bool profile = false;
    std::vector<cudaEvent_t> ev;          // SPH_NPHASES + 1 events per profiled step
    double prof_ms[SPH_NPHASES] = {};
    uint64_t prof_steps = 0;
    // differentiable mode: checkpoints every ckpt_every steps since
    // sph_diff_begin, the tape of one segment and the adjoint arrays
    bool diff = false;
    uint32_t ckpt_every = 0;
    uint64_t diff_steps = 0;
    int64_t relayout_saved = 0;
    struct Ckpt {
        int a;
        double t_host;
        char *buf;
    };
    std::vector<Ckpt> ckpts;
    // checkpoint buffers handed back by sph_diff_end and the backward, kept
    // for the next forward of a calibration loop; freed by sph_destroy
    std::vector<char *> ckpt_pool;
    // Darcy flow, on after sph_darcy_upload; the current pressure buffer is
    // darcy.H[a ^ dflip] (both flip once per step)
    bool darcy_on = false;
    DarcyDev darcy{};
    // in the step graphs the Darcy kernels run on a branch beside the force
    // and wall kernels: forked after the cell list, joined at the step's end
    cudaStream_t darcy_stream = nullptr;
    cudaEvent_t darcy_fork = nullptr, darcy_join = nullptr;
    // in the step graphs the wall reduction and integration of a step run on
    // a branch forked after its force kernel and joined before the next
    // step's force kernel (or the graph's end); wall_pending: a fork is open
    cudaStream_t wall_stream = nullptr;
    cudaEvent_t wall_fork = nullptr, wall_join = nullptr;
    bool wall_pending = false;
    ForceConsts graph_fc{};          // the force kernel's constants in the step graphs
    int dflip = 0;
    double mean_radius = 0.0;        // of the uploaded particles, summed in caller order
    // ray tracer scratch: per-pixel keys and image, per-particle values
    void *rt_buf = nullptr;
    size_t rt_bytes = 0;
    size_t ckpt_bytes = 0;                // size of one pooled buffer
    cudaEvent_t ckpt_ev = nullptr;        // orders a checkpoint copy against the caller's stream
    std::vector<void *> diff_allocs;
    size_t diff_bytes = 0;
    double *bwd_scratch = nullptr;        // the backward's seeds and results, 13 np doubles
    AdjDev adj{};
    // graphs of one segment's re-run with the tape and of its reverse, by
    // (segment length, starting buffer)
    std::map<std::pair<int, int>, cudaGraphExec_t> diff_graphs;
};

namespace {

int fail(sph_ctx *c, int code, const std::string &msg)
{
    if (c) {
        c->err = msg;
        if (c->sticky == SPH_OK && code != SPH_ERR_BAD_INPUT) c->sticky = code;
    }
    return code;
}

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(c, SPH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int dalloc(sph_ctx *c, T **p, size_t count, std::vector<void *> *owner = nullptr)
{
    const size_t bytes = sizeof(T) * (count ? count : 1);
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return fail(c, SPH_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    e = cudaMemsetAsync(q, 0, bytes, c->stream);
    if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    (owner ? owner : &c->allocs)->push_back(q);
    (owner ? c->diff_bytes : c->device_bytes) += bytes;
    *p = static_cast<T *>(q);
    return SPH_OK;
}

int status_to_code(uint32_t st)
{
    if (st & ST_NC_OVERFLOW) return SPH_ERR_NC_OVERFLOW;
    if (st & ST_OUT_OF_GRID) return SPH_ERR_OUT_OF_GRID;
    if (st & ST_TIMEOUT) return SPH_ERR_TIMEOUT;
    if (st & ST_BOND_ALIAS) return SPH_ERR_BOND_ALIAS;
    return SPH_OK;
}

const char *status_msg(int code)
{
    switch (code) {
    case SPH_ERR_NC_OVERFLOW: return "a particle has more than 32 contacts (NC overflow)";
    case SPH_ERR_OUT_OF_GRID:
        return "one or more particles moved outside the grid; is the time step too large?";
    case SPH_ERR_TIMEOUT: return "a bounded device wait gave up";
    case SPH_ERR_BOND_ALIAS: return "a bond broke while nb0 < np: its marker aliases particle nb0";
    default: return "";
    }
}

// ---- host -> device conversion kernels -------------------------------------
// The caller's rows are copied as they are into device staging and repacked
// here, so a pinned host buffer goes over the bus at full speed and the host
// runs no per-particle loop.  At upload, storage order is the caller's order.

// four-double host rows: the first three into `dst`, the fourth into lane
// `lane` of w_user
__global__ void k_user_to_p3(const double4 *src, P3 *dst, double *w, int lane, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = src[i];
    dst[i] = P3{v.x, v.y, v.z};
    w[WLANES * (size_t)i + lane] = v.w;
}

// the fixvel flag of the integration (vel.w > 0)
__global__ void k_fixed_flags(const double4 *vel, uint8_t *fixed, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) fixed[i] = vel[i].w > 0.0f ? 1 : 0;
}

// acc / angacc rows with their unused fourth lane cleared
__global__ void k_rows_zero_w(const double4 *src, double4 *dst, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 v = src[i];
    dst[i] = make_double4(v.x, v.y, v.z, 0.0);
}

// planar es, ev into the interleaved esv rows
__global__ void k_pack2(const double *a, const double *b, double2 *dst, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_double2(a[i], b[i]);
}

// planar es_dot, ev_dot, p into the edp rows
__global__ void k_pack3(const double *a, const double *b, const double *c, double4 *dst, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = make_double4(a[i], b[i], c[i], 0.0);
}

// the identity storage order of an upload
__global__ void k_iota3(uint32_t *a, uint32_t *b, uint32_t *c, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = i;
    b[i] = i;
    c[i] = i;
}

// ---- device -> host conversion kernels ------------------------------------
template <typename T>
__global__ void k_to_user(const T *src, T *dst, const uint32_t *sidx, uint32_t n)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < n) dst[u] = src[sidx[u]];
}

// a three-double row and its kept fourth lane, as the host's four-double row
__global__ void k_p3_to_user(const P3 *src, const double *w, int lane, double4 *dst,
                             const uint32_t *sidx, uint32_t n)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const P3 v = src[sidx[u]];
    dst[u] = make_double4(v.x, v.y, v.z, w[WLANES * (size_t)u + lane]);
}

// one lane of interleaved rows (esv, edp) in caller order, planar
template <typename T, int K>
__global__ void k_lane_to_user(const T *src, double *dst, const uint32_t *sidx, uint32_t n)
{
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const T v = src[sidx[u]];
    dst[u] = reinterpret_cast<const double *>(&v)[K];
}

__global__ void k_rows_to_user(Dev d, uint32_t *contacts, double4 *distmod, double4 *delta_t,
                               int A)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)d.np_all * NC) return;
    const uint32_t u = (uint32_t)(e / NC), i = (uint32_t)(e % NC);
    const uint32_t s = d.sidx[u];
    const Params &P = prm_of(d, s);
    const bool occ = (d.cmask[s] >> i) & 1u;
    const uint32_t v = d.contacts[tile_at(s, i, NC)];
    // partners as indices within the particle's own scene; np marks empty
    if (contacts) contacts[e] = occ ? d.uid[v] - P.uid_base : P.np;
    if (distmod) {
        double4 o = make_double4(0.0, 0.0, 0.0, 0.0);
        if (occ) {
            const ulonglong2 c = d.dmc[s];
            const uint32_t code = (uint32_t)((i < 16 ? (c.x >> (4 * i)) : (c.y >> (4 * (i - 16)))) & 0xFull);
            const d3 dm = decode_dm(code, P);
            o = make_double4(dm.x, dm.y, dm.z, d.xr[A][v].w);
        }
        distmod[e] = o;
    }
    if (delta_t) {
        // the reference writes the history's fourth lane as 0 (contactmodels.cuh:487, :664)
        const P3 v3 = d.delta_t[tile_at(s, i, NC)];
        delta_t[e] = occ ? make_double4(v3.x, v3.y, v3.z, 0.0) : make_double4(0.0, 0.0, 0.0, 0.0);
    }
}

__global__ void k_cells_out(Dev d, uint32_t *cell_sorted, uint32_t *perm, uint32_t *cstart,
                            uint32_t *cend)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d.ncells_all) {
        const uint32_t b = d.cell_start[i], e = d.cell_start[i + 1];
        cstart[i] = (b == e) ? 0xffffffffu : b;
        cend[i] = (b == e) ? 0u : e;
        for (uint32_t k = b; k < e; ++k) cell_sorted[k] = i;
    }
    if (i == d.ncells_all) {
        for (uint32_t k = d.cell_start[i]; k < d.cell_start[i + 1]; ++k) cell_sorted[k] = 0xffffffffu;
    }
    if (i < d.np_all) perm[i] = d.uid[d.cellorder[i]];
}

__global__ void k_count_contacts(const uint32_t *cmask, uint32_t np, unsigned long long *out)
{
    uint32_t acc = 0;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < np; s += gridDim.x * blockDim.x)
        acc += __popc(cmask[s]);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31u) == 0 && acc) atomicAdd(out, (unsigned long long)acc);
}

int sync_status(sph_ctx *c)
{
    CK(cudaStreamSynchronize(c->stream));
    uint32_t st = 0;
    CK(cudaMemcpyAsync(&st, c->d.status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
    const int code = status_to_code(st);
    if (code != SPH_OK) return fail(c, code, status_msg(code));
    return SPH_OK;
}

// Inside a stream capture: the rebuild as a conditional node whose body the
// side stream captures, gated by k_rebuild_gate.
int capture_rebuild_conditional(sph_ctx *c, int a, cudaStream_t st)
{
    cudaStreamCaptureStatus cs;
    unsigned long long id;
    cudaGraph_t g;
    const cudaGraphNode_t *deps;
    size_t nd;
    CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    launch_rebuild_gate(h, c->d.rebuild, st);
    CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(c->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    launch_rebuild(c->d, c->np_all, c->ncells_all, a, c->side);
    CK(cudaStreamEndCapture(c->side, &body));
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return SPH_OK;
}

int enqueue_one_step(sph_ctx *c, int a, int write_outputs, cudaStream_t st, bool capturing = false)
{
    if (capturing && c->cond_rebuild) {
        const int rc = capture_rebuild_conditional(c, a, st);
        if (rc != SPH_OK) return rc;
    } else {
        launch_rebuild(c->d, c->np_all, c->ncells_all, a, st);
    }
    launch_bonds(c->d, c->hp, c->hp.nb0, a, st);
    // The Darcy block reads the step's start positions (buffer a) and its
    // cell list, which nothing changes before the next step's rebuild, and
    // writes only the fluid grid: in a graph it runs beside the force and
    // wall kernels and joins before the step ends.
    const bool branch = capturing && c->darcy_on && c->darcy_stream;
    if (branch) {
        CK(cudaEventRecord(c->darcy_fork, st));
        CK(cudaStreamWaitEvent(c->darcy_stream, c->darcy_fork, 0));
        launch_darcy(c->d, c->darcy, c->hp, a, a ^ c->dflip, c->darcy_stream);
        CK(cudaEventRecord(c->darcy_join, c->darcy_stream));
    }
    const int model = (int)c->hp.contactmodel;
    launch_topo(c->d, c->np_all, model == 1, a, st);
    launch_contact(c->d, c->hp, c->np_all, model, a, write_outputs, st);
    if (c->wall_pending) {
        // the walls moved by the previous step's branch, before this step's
        // wall forces read them
        CK(cudaStreamWaitEvent(st, c->wall_join, 0));
        c->wall_pending = false;
    }
    launch_force(c->d, c->hp, c->np_all, model, a, write_outputs, st);
    if (c->darcy_on && !branch) launch_darcy(c->d, c->darcy, c->hp, a, a ^ c->dflip, st);
    if (capturing && c->hp.nw > 0 && !c->batched) {
        CK(cudaEventRecord(c->wall_fork, st));
        CK(cudaStreamWaitEvent(c->wall_stream, c->wall_fork, 0));
        launch_wall_motion(c->d, c->np_all, c->wall_stream);
        CK(cudaEventRecord(c->wall_join, c->wall_stream));
        c->wall_pending = true;
        launch_tail(c->d, st);
    } else {
        launch_walls(c->d, c->np_all, c->hp.nw, st);
    }
    if (branch) CK(cudaStreamWaitEvent(st, c->darcy_join, 0));
    return SPH_OK;
}

int capture(sph_ctx *c, cudaGraphExec_t *out, int a, int nsteps, int write_last)
{
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int aa = a;
    int rc = SPH_OK;
    c->wall_pending = false;
    for (int i = 0; i < nsteps && rc == SPH_OK; ++i) {
        rc = enqueue_one_step(c, aa, (write_last && i == nsteps - 1) ? 1 : 0, c->stream, true);
        aa ^= 1;
    }
    if (c->wall_pending) {
        // the last step's walls are part of the graph's work (and a capture
        // that failed ends with its branch joined)
        const cudaError_t e = cudaStreamWaitEvent(c->stream, c->wall_join, 0);
        if (e != cudaSuccess && rc == SPH_OK)
            rc = fail(c, SPH_ERR_CUDA, std::string("wall join: ") + cudaGetErrorString(e));
    }
    c->wall_pending = false;
    if (rc != SPH_OK) {
        // conditional nodes unavailable: end the broken capture and capture
        // the plain rebuild instead
        cudaStreamEndCapture(c->stream, &g);
        if (g) cudaGraphDestroy(g);
        if (c->side) cudaStreamEndCapture(c->side, &g);
        cudaGetLastError();
        if (!c->cond_rebuild) return rc;
        c->cond_rebuild = false;
        c->sticky = SPH_OK;
        c->err.clear();
        return capture(c, out, a, nsteps, write_last);
    }
    CK(cudaStreamEndCapture(c->stream, &g));
    cudaError_t e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return fail(c, SPH_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return SPH_OK;
}

void drop_graphs(sph_ctx *c)
{
    for (auto &g : c->g_multi)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    for (auto &row : c->g_single)
        for (auto &g : row)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    c->graphs_for_k = 0;
}

int ensure_graphs(sph_ctx *c)
{
    // graphs carry the force kernel's constants: an upload that changed one
    // (the skin, esv_skip) captures them again
    const ForceConsts fc = force_consts(c->hp);
    if (c->graphs_for_k == c->graph_steps && c->g_single[0][0] &&
        std::memcmp(&fc, &c->graph_fc, sizeof(fc)) == 0)
        return SPH_OK;
    drop_graphs(c);
    for (int a = 0; a < 2; ++a) {
        int rc;
        if ((rc = capture(c, &c->g_multi[a], a, c->graph_steps, 0)) != SPH_OK) return rc;
        for (int w = 0; w < 2; ++w)
            if ((rc = capture(c, &c->g_single[a][w], a, 1, w)) != SPH_OK) return rc;
    }
    c->graphs_for_k = c->graph_steps;
    c->graph_fc = force_consts(c->hp);
    return SPH_OK;
}

// profile mode: one step with events between the phases
int profiled_step(sph_ctx *c, int a, int write_outputs, cudaStream_t st)
{
    if (c->ev.empty()) {
        c->ev.resize(SPH_NPHASES + 1);
        for (auto &e : c->ev) CK(cudaEventCreate(&e));
    }
    // the phases in launch order; event k + 1 closes order[k]
    static const int order[SPH_NPHASES] = {SPH_PHASE_CELLS, SPH_PHASE_BONDS, SPH_PHASE_TOPO,
                                           SPH_PHASE_CONTACT, SPH_PHASE_FORCE, SPH_PHASE_WALLS,
                                           SPH_PHASE_DARCY};
    CK(cudaEventRecord(c->ev[0], st));
    launch_rebuild(c->d, c->np_all, c->ncells_all, a, st);
    CK(cudaEventRecord(c->ev[1], st));
    launch_bonds(c->d, c->hp, c->hp.nb0, a, st);
    CK(cudaEventRecord(c->ev[2], st));
    launch_topo(c->d, c->np_all, c->hp.contactmodel == 1, a, st);
    CK(cudaEventRecord(c->ev[3], st));
    launch_contact(c->d, c->hp, c->np_all, (int)c->hp.contactmodel, a, write_outputs, st);
    CK(cudaEventRecord(c->ev[4], st));
    launch_force(c->d, c->hp, c->np_all, (int)c->hp.contactmodel, a, write_outputs, st);
    CK(cudaEventRecord(c->ev[5], st));
    launch_walls(c->d, c->np_all, c->hp.nw, st);
    CK(cudaEventRecord(c->ev[6], st));
    if (c->darcy_on) launch_darcy(c->d, c->darcy, c->hp, a, a ^ c->dflip, st);
    CK(cudaEventRecord(c->ev[7], st));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(c->ev[7]));
    for (int k = 0; k < SPH_NPHASES; ++k) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev[k], c->ev[k + 1]));
        c->prof_ms[order[k]] += ms;
    }
    c->prof_steps++;
    return SPH_OK;
}

int do_relayout(sph_ctx *c, cudaStream_t st)
{
    // the cell list must describe the current positions before storage follows it
    launch_rebuild(c->d, c->np_all, c->ncells_all, c->a, st);
    relayout(c->d, c->np_all, c->a, c->scratch, st);
    // the bonds follow their particles' new storage indices
    if (!c->batched) launch_bond_storage(c->d, c->hp.nb0, c->np_all, st);
    // the slot rows moved: every chunk may hold a contact until the next
    // force pass has looked
    CK(cudaMemsetAsync(c->d.cflag, 1, div_up(c->np_all, 32), st));
    CK(cudaMemsetAsync(c->d.settled, 0, c->np_all, st));
    CK(cudaGetLastError());
    c->relayouts++;
    c->since_relayout = 0;
    return SPH_OK;
}

}  // namespace

extern "C" {

int sph_version(void) { return SPHK_VERSION; }

const char *sph_last_error(const sph_ctx *c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"

namespace {

// The reasons a scene configuration is refused (empty when it is valid).
std::string config_problem(const sph_config *cfg)
{
    const uint64_t ncells = (uint64_t)cfg->num[0] * cfg->num[1] * cfg->num[2];
    if (cfg->np == 0) return "np must be positive";
    if (cfg->nw > SPHK_MAXWALLS) return "nw exceeds MAXWALLS (6)";
    if (ncells == 0 || ncells >= 0xfffffff0ull) return "grid.num must be positive and below 2^32 cells";
    if (cfg->contactmodel < 1 || cfg->contactmodel > 3) return "contact model must be 1, 2 or 3";
    if (!(cfg->dt > 0.0)) return "dt must be positive";
    if ((uint64_t)cfg->np * NC >= 0xffffffffull) return "np too large";
    return "";
}

// Params of one scene (the rest -- rmax, skin -- is set at upload).
void fill_params(const sph_config *cfg, Params &P)
{
    P = Params{};
    P.np = cfg->np; P.nw = cfg->nw; P.nb0 = cfg->nb0; P.contactmodel = cfg->contactmodel;
    P.periodic = cfg->periodic;
    double ext = 0.0;
    for (int k = 0; k < 3; ++k) {
        P.num[k] = cfg->num[k];
        P.origo[k] = cfg->origo[k];
        P.L[k] = cfg->L[k];
        P.cellsize[k] = cfg->L[k] / (double)cfg->num[k];
        P.g[k] = cfg->g[k];
        ext = std::fmax(ext, std::fmax(std::fabs(cfg->origo[k]), std::fabs(cfg->L[k])));
    }
    P.ncells = cfg->num[0] * cfg->num[1] * cfg->num[2];
    P.dt = cfg->dt;
    P.k_n = cfg->k_n; P.k_t = cfg->k_t; P.k_r = cfg->k_r;
    P.gamma_n = cfg->gamma_n; P.gamma_t = cfg->gamma_t; P.gamma_r = cfg->gamma_r;
    P.mu_s = cfg->mu_s; P.mu_d = cfg->mu_d; P.mu_r = cfg->mu_r;
    P.gamma_wn = cfg->gamma_wn; P.gamma_wt = cfg->gamma_wt;
    P.mu_ws = cfg->mu_ws; P.mu_wd = cfg->mu_wd; P.rho = cfg->rho;
    P.kappa = cfg->kappa; P.db = cfg->db; P.V_b = cfg->V_b;
    P.lambda_bar = cfg->lambda_bar; P.sigma_b = cfg->sigma_b; P.tau_b = cfg->tau_b;
    P.devs_A = cfg->devs_A; P.devs_f = cfg->devs_f;
    for (int k = 0; k < MAXWALLS; ++k) P.wmode[k] = cfg->wmode[k];
    // float rounding of coordinates is below 2^-24 |x|; particles near the
    // domain stay within a few domain extents, so 1e-6 * 4 * extent is a
    // generous bound on the cull's absolute error
    P.cull_eps = (float)(4e-6 * (ext > 0.0 ? ext : 1.0));
    P.prune_pad = 4.0 * (double)P.cull_eps;
    // model 1 also acts on pairs with a gap below db (capillary cohesion)
    P.reach_extra = (cfg->contactmodel == 1 && cfg->db > 0.0) ? cfg->db : 0.0;
}

// One context over `ninst` scenes laid end to end: particle u of scene i is
// global particle uid_base(i) + u, its cells are global cells cell_base(i)..
int create_impl(const sph_config *cfgs, uint32_t ninst, bool batched, sph_ctx **out)
{
    sph_ctx *c = new sph_ctx();
    *out = c;
    uint64_t np_all = 0, ncells_all = 0, nb0 = 0;
    for (uint32_t i = 0; i < ninst; ++i) {
        const sph_config *cfg = &cfgs[i];
        std::string why = config_problem(cfg);
        if (why.empty() && batched) {
            if (cfg->contactmodel != 2) why = "batched scenes use contact model 2";
            else if (cfg->nw != 0) why = "batched scenes have no dynamic walls (nw = 0)";
            else if (cfg->nb0 != 0) why = "batched scenes have no bonds (nb0 = 0)";
            else if (cfg->device != cfgs[0].device) why = "batched scenes share one device";
        }
        if (!why.empty()) {
            c->err = batched ? "scene " + std::to_string(i) + ": " + why : why;
            return SPH_ERR_BAD_INPUT;
        }
        np_all += cfg->np;
        ncells_all += (uint64_t)cfg->num[0] * cfg->num[1] * cfg->num[2];
        nb0 += cfg->nb0;
    }
    if (np_all * NC >= 0xffffffffull || ncells_all >= 0xfffffff0ull) {
        c->err = "the scenes together are too large for one context";
        return SPH_ERR_BAD_INPUT;
    }
    c->batched = batched;
    c->ninst = ninst;
    c->np_all = (uint32_t)np_all;
    c->ncells_all = (uint32_t)ncells_all;
    c->hps.resize(ninst);
    uint32_t cb = 0, ub = 0;
    std::vector<uint32_t> cell_bases(ninst + 1);
    for (uint32_t i = 0; i < ninst; ++i) {
        fill_params(&cfgs[i], c->hps[i]);
        c->hps[i].cell_base = cb;
        c->hps[i].uid_base = ub;
        cell_bases[i] = cb;
        cb += c->hps[i].ncells;
        ub += c->hps[i].np;
    }
    cell_bases[ninst] = cb;
    c->hp = c->hps[0];
    c->device = cfgs[0].device;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->wall_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->wall_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->wall_join, cudaEventDisableTiming));

    const size_t np = c->np_all;
    const size_t ncells = c->ncells_all;
    Dev &d = c->d;
    d.np_all = c->np_all;
    d.ncells_all = c->ncells_all;
    d.ninst = ninst;
    int rc = SPH_OK;
#define AL(ptr, n) if ((rc = dalloc(c, &(ptr), (n))) != SPH_OK) return rc;
    // the rows the force kernel copies in tiles, in whole tiles
    const size_t npad = padded_rows(np);
    for (int b = 0; b < 2; ++b) {
        AL(d.xr[b], npad); AL(d.vel[b], npad); AL(d.angvel[b], npad); AL(d.xs[b], np);
    }
    AL(d.vel0, npad); AL(d.angvel0, npad); AL(d.angpos, npad); AL(d.xysum, npad); AL(d.esv, np);
    AL(d.w_user, WLANES * np); AL(d.fixed, npad);
    AL(d.force, np); AL(d.torque, np); AL(d.acc, np); AL(d.angacc, np); AL(d.edp, np);
    AL(d.uid, np); AL(d.sidx, np); AL(d.cell, npad); AL(d.outside, np);
    AL(d.contacts, tiled_size(np, NC)); AL(d.dmc, np); AL(d.delta_t, tiled_size(np, NC));
    AL(d.cmask, np);
    AL(d.cflag, div_up(np, 32));
    AL(d.cell_start, ncells + 2); AL(d.cellorder, np); AL(d.pos, npad); AL(d.cell_fill, ncells + 1);
    AL(d.scan_tiles, scan_tile_count(c->ncells_all));
    AL(d.alias_any, 1);
    AL(d.vl, tiled_size(np, VL_CAP)); AL(d.vl_meta, tiled_size(np, VL_CAP)); AL(d.vl_len, np);
    AL(d.disp, npad);
    AL(d.vl_gap, np); AL(d.settled, np);
    AL(d.movers, MOVER_CAP); AL(d.dirty, ncells + 1); AL(d.vs, 1);
    AL(d.wf_pp, np); AL(d.wtouch, npad); AL(d.wf_partial, div_up(np, 256));
    AL(d.wf_flag, div_up(np, 256));
    AL(d.walls, 1);
    AL(d.bonds, nb0); AL(d.bonds_delta, nb0); AL(d.bonds_omega, nb0);
    AL(d.bond_f, nb0); AL(d.bond_t, nb0); AL(d.bond_xu, nb0); AL(d.bond_s, nb0);
    AL(d.bond_ptr, np + 1); AL(d.bond_list, 2 * (size_t)nb0);
    if (c->hp.contactmodel == 1) {
        AL(d.c1acc, np);
    } else {
        AL(d.csum_f, np); AL(d.csum_t, np); AL(d.csum_es, np);
    }
    AL(d.status, 1); AL(d.rebuild, 1); AL(d.prm, ninst);
    if (batched) {
        AL(d.inst, np);
        AL(d.inst_cell_base, (size_t)ninst + 1);
        CK(cudaMemcpyAsync(d.inst_cell_base, cell_bases.data(), ((size_t)ninst + 1) * 4,
                      cudaMemcpyHostToDevice, c->stream));
    }
    c->scratch_bytes = tiled_size(np, NC) * sizeof(P3) + np * sizeof(uint32_t) + 256;
    char *sc = nullptr;
    AL(sc, c->scratch_bytes);
    c->scratch = sc;
#undef AL
    CK(cudaMemcpyAsync(d.prm, c->hps.data(), sizeof(Params) * ninst, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    // The step graphs depend only on what is fixed here (sizes, device
    // pointers, contact model, walls, bonds); every value an upload changes
    // is read from device memory.  Capturing them now puts their cost in
    // context creation rather than in the first sph_step.  A later change of
    // SPH_OPT_GRAPH_STEPS, or the Darcy flow, captures them again.
    if (!batched) return ensure_graphs(c);
    return SPH_OK;
}

}  // namespace

extern "C" {

int sph_create(const sph_config *cfg, sph_ctx **out)
{
    if (!cfg || !out) return SPH_ERR_BAD_INPUT;
    return create_impl(cfg, 1, false, out);
}

int sph_batch_create(const sph_config *cfgs, uint32_t ninst, sph_ctx **out)
{
    if (!cfgs || !out || ninst == 0) return SPH_ERR_BAD_INPUT;
    return create_impl(cfgs, ninst, true, out);
}

int sph_set_option(sph_ctx *c, int option, int64_t value)
{
    if (!c) return SPH_ERR_BAD_INPUT;
    if (option == SPH_OPT_RELAYOUT_EVERY && value >= 0) {
        c->relayout_every = value;
        return SPH_OK;
    }
    if (option == SPH_OPT_VERLET_SKIN && value >= 0 && value <= 1000) {
        if (c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "set the Verlet skin before sph_upload");
        c->skin_rel = (double)value / 1000.0;
        return SPH_OK;
    }
    if (option == SPH_OPT_PROFILE && (value == 0 || value == 1)) {
        c->profile = value != 0;
        return SPH_OK;
    }
    if (option == SPH_OPT_GRAPH_STEPS && value >= 1 && value <= 64) {
        c->graph_steps = (int)value;
        return SPH_OK;
    }
    if (option == SPH_OPT_BLOCK_SHAPES && (value == 0 || value == 1)) {
        // kernels and graphs take Dev by value: capture again with the shape
        if (c->d.shape != (uint32_t)value) {
            CK(cudaSetDevice(c->device));
            CK(cudaStreamSynchronize(c->stream));
            c->d.shape = (uint32_t)value;
            drop_graphs(c);
            if (!c->batched) return ensure_graphs(c);
        }
        return SPH_OK;
    }
    if (option == SPH_OPT_TOPO_SPAN && (value == 0 || value == 1 || value == 2 || value == 4)) {
        if (c->d.topo_span != (uint32_t)value) {
            CK(cudaSetDevice(c->device));
            CK(cudaStreamSynchronize(c->stream));
            c->d.topo_span = (uint32_t)value;
            drop_graphs(c);
            if (!c->batched) return ensure_graphs(c);
        }
        return SPH_OK;
    }
    return fail(c, SPH_ERR_BAD_INPUT, "unknown option or value");
}

int sph_upload(sph_ctx *c, const sph_host_state *h)
{
    if (!c || !h || !h->x || !h->vel || !h->xysum || !h->force || !h->angpos || !h->angvel ||
        !h->torque || !h->es_dot || !h->es || !h->ev_dot || !h->ev || !h->p)
        return fail(c, SPH_ERR_BAD_INPUT, "sph_upload: missing required array");
    const Params &P = c->hp;
    if (P.nw > 0 && (!h->walls_nx || !h->walls_mvfd))
        return fail(c, SPH_ERR_BAD_INPUT, "sph_upload: walls_nx/walls_mvfd required when nw > 0");
    if (P.nb0 > 0 && (!h->bonds || !h->bonds_delta || !h->bonds_omega))
        return fail(c, SPH_ERR_BAD_INPUT, "sph_upload: bond arrays required when nb0 > 0");
    CK(cudaSetDevice(c->device));
    const size_t np = c->np_all, nb0 = P.nb0;
    Dev &d = c->d;
    const int A = 0;
    // the Darcy pressure buffers keep their roles across the parity reset;
    // graphs hold the buffer of each step, so they are captured again
    if (c->darcy_on && c->a != A) drop_graphs(c);
    c->dflip ^= c->a ^ A;
    c->a = A;
    {
        // meanRadius (src/darcy.cpp:646-653) for the Darcy grain-size factor
        double r_sum = 0.0;
        for (size_t i = 0; i < np; ++i) r_sum += h->x[4 * i + 3];
        c->mean_radius = r_sum / (double)np;
    }
    // scene of every particle (particles of scene i follow those of scene i-1),
    // for batched contexts and for contact rows given by the caller
    std::vector<uint32_t> inst_of;
    if (c->batched || h->contacts) {
        inst_of.assign(np, 0u);
        for (uint32_t i = 0; i < c->ninst; ++i)
            for (uint32_t u = 0; u < c->hps[i].np; ++u) inst_of[c->hps[i].uid_base + u] = i;
    }
    if (c->batched) CK(cudaMemcpyAsync(d.inst, inst_of.data(), np * 4, cudaMemcpyHostToDevice, c->stream));
    // kinematics (identity storage order for now)
    CK(cudaMemcpyAsync(d.xr[A], h->x, np * 32, cudaMemcpyHostToDevice, c->stream));
    {
        // largest radius of each scene, for the cell-level distance test of
        // contact search; one Verlet skin for the whole context, from the
        // largest radius of all
        double rmax_all = 0.0;
        for (uint32_t i = 0; i < c->ninst; ++i) {
            Params &Q = c->hps[i];
            double rmax = 0.0;
            for (size_t u = Q.uid_base; u < (size_t)Q.uid_base + Q.np; ++u)
                rmax = std::fmax(rmax, h->x[4 * u + 3]);
            Q.rmax = rmax;
            rmax_all = std::fmax(rmax_all, rmax);
        }
        for (auto &Q : c->hps) Q.skin = c->skin_rel * rmax_all;
        // a zero energy rate may skip the es/ev update only if no sum is -0.0
        bool negzero = false;
        for (size_t i = 0; i < np && !negzero; ++i)
            negzero = (h->es[i] == 0.0 && std::signbit(h->es[i])) ||
                      (h->ev[i] == 0.0 && std::signbit(h->ev[i]));
        for (auto &Q : c->hps) Q.esv_skip = negzero ? 0u : 1u;
        c->hp = c->hps[0];
        CK(cudaMemcpyAsync(d.prm, c->hps.data(), sizeof(Params) * c->ninst, cudaMemcpyHostToDevice, c->stream));
        Verlet V{};
        V.step = 1;
        V.all_rebuild = 1;
        CK(cudaMemcpyAsync(d.vs, &V, sizeof(V), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemsetAsync(d.dirty, 0, ((size_t)c->ncells_all + 1) * sizeof(uint32_t), c->stream));
        CK(cudaMemsetAsync(d.vl_len, VL_NONE, np, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    {
        // vel, angvel, vel0, angvel0, angpos: three doubles on the device, the
        // fourth lane kept by caller index for the download; fixvel > 0 as a
        // flag for the integration
        // the caller's rows go to device staging as they are and are
        // repacked there (stream order serialises the reuse of the staging)
        cudaStream_t st = c->stream;
        const unsigned g = div_up(np, 256);
        double4 *stage = static_cast<double4 *>(c->scratch);
        const double *src[WLANES];
        P3 *dst[WLANES];
        src[W_VEL0] = h->vel0 ? h->vel0 : h->vel;
        src[W_ANGVEL0] = h->angvel0 ? h->angvel0 : h->angvel;
        src[W_ANGPOS] = h->angpos;
        src[W_ANGVEL] = h->angvel;
        src[W_VEL] = h->vel;
        dst[W_VEL0] = d.vel0;
        dst[W_ANGVEL0] = d.angvel0;
        dst[W_ANGPOS] = d.angpos;
        dst[W_ANGVEL] = d.angvel[A];
        dst[W_VEL] = d.vel[A];
        for (int f = 0; f < WLANES; ++f) {
            CK(cudaMemcpyAsync(stage, src[f], np * 32, cudaMemcpyHostToDevice, st));
            k_user_to_p3<<<g, 256, 0, st>>>(stage, dst[f], d.w_user, f, (uint32_t)np);
            if (f == W_VEL) k_fixed_flags<<<g, 256, 0, st>>>(stage, d.fixed, (uint32_t)np);
        }
        CK(cudaMemcpyAsync(d.force, h->force, np * 32, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(d.torque, h->torque, np * 32, cudaMemcpyHostToDevice, st));
        const std::pair<const double *, double4 *> accs[] = {{h->acc, d.acc}, {h->angacc, d.angacc}};
        for (const auto &a : accs) {
            if (a.first) {
                CK(cudaMemcpyAsync(stage, a.first, np * 32, cudaMemcpyHostToDevice, st));
                k_rows_zero_w<<<g, 256, 0, st>>>(stage, a.second, (uint32_t)np);
            } else {
                CK(cudaMemsetAsync(a.second, 0, np * 32, st));
            }
        }
        CK(cudaMemcpyAsync(d.xysum, h->xysum, np * 16, cudaMemcpyHostToDevice, st));
        double *planar = reinterpret_cast<double *>(stage);
        CK(cudaMemcpyAsync(planar, h->es, np * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(planar + np, h->ev, np * 8, cudaMemcpyHostToDevice, st));
        k_pack2<<<g, 256, 0, st>>>(planar, planar + np, d.esv, (uint32_t)np);
        CK(cudaMemcpyAsync(planar, h->es_dot, np * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(planar + np, h->ev_dot, np * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(planar + 2 * np, h->p, np * 8, cudaMemcpyHostToDevice, st));
        k_pack3<<<g, 256, 0, st>>>(planar, planar + np, planar + 2 * np, d.edp, (uint32_t)np);
        k_iota3<<<g, 256, 0, st>>>(d.uid, d.sidx, d.cellorder, (uint32_t)np);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
    }
    // contact slots: partners, periodic-shift codes, occupancy, history
    if (!h->contacts) {
        // the reference's initial state: every slot empty, zero history
        CK(cudaMemsetAsync(d.contacts, 0xff, tiled_size(np, NC) * 4, c->stream));   // empty slots are read through cmask only
        CK(cudaMemsetAsync(d.dmc, 0, np * 16, c->stream));
        CK(cudaMemsetAsync(d.cmask, 0, np * 4, c->stream));
        CK(cudaMemsetAsync(d.delta_t, 0, tiled_size(np, NC) * sizeof(P3), c->stream));
    } else {
        // the caller's rows [np][NC] into tiles; the history's fourth lane is
        // not kept (the reference writes it as 0)
        std::vector<uint32_t> rows(tiled_size(np, NC), (uint32_t)np);
        std::vector<unsigned long long> dmc(np * 2, 0ull);
        std::vector<uint32_t> cmask(np, 0u);
        std::vector<double> dts(tiled_size(np, NC) * 3, 0.0);
        for (size_t i = 0; i < np; ++i) {
            // partners are indices within the particle's own scene
            const Params &Q = c->hps[inst_of[i]];
            for (int k = 0; k < NC; ++k) {
                const uint32_t v = h->contacts[i * NC + k];
                if (v >= Q.np) continue;
                const size_t at = tile_at((uint32_t)i, (uint32_t)k, NC);
                rows[at] = v + Q.uid_base;
                cmask[i] |= 1u << k;
                uint32_t code = 0;
                if (h->distmod) {
                    const double dx = h->distmod[(i * NC + k) * 4];
                    const double dy = h->distmod[(i * NC + k) * 4 + 1];
                    if (dx == Q.L[0]) code |= 1u; else if (dx == -Q.L[0]) code |= 2u;
                    else if (dx != 0.0) return fail(c, SPH_ERR_BAD_INPUT, "distmod.x must be 0 or +-L[0]");
                    if (dy == Q.L[1]) code |= 4u; else if (dy == -Q.L[1]) code |= 8u;
                    else if (dy != 0.0) return fail(c, SPH_ERR_BAD_INPUT, "distmod.y must be 0 or +-L[1]");
                }
                dmc[2 * i + (k >> 4)] |= (unsigned long long)code << (4 * (k & 15));
                if (h->delta_t)
                    for (int q = 0; q < 3; ++q) dts[at * 3 + q] = h->delta_t[(i * NC + k) * 4 + q];
            }
        }
        CK(cudaMemcpyAsync(d.contacts, rows.data(), rows.size() * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(d.dmc, dmc.data(), np * 16, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(d.cmask, cmask.data(), np * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(d.delta_t, dts.data(), dts.size() * 8, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));   // the host rows above go out of scope
    }
    // walls
    {
        Walls W{};
        for (uint32_t k = 0; k < P.nw; ++k) {
            W.nx[k] = make_double4(h->walls_nx[4 * k], h->walls_nx[4 * k + 1], h->walls_nx[4 * k + 2], h->walls_nx[4 * k + 3]);
            W.mvfd[k] = make_double4(h->walls_mvfd[4 * k], h->walls_mvfd[4 * k + 1], h->walls_mvfd[4 * k + 2], h->walls_mvfd[4 * k + 3]);
            W.vel0[k] = h->walls_vel0 ? h->walls_vel0[k] : h->walls_mvfd[4 * k + 1];
        }
        W.t_current = h->t_current;
        W.done_blocks = 0;
        CK(cudaMemcpyAsync(d.walls, &W, sizeof(W), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    CK(cudaMemsetAsync(d.wf_pp, 0, np * sizeof(double), c->stream));
    CK(cudaMemsetAsync(d.wtouch, 0, np, c->stream));
    CK(cudaMemsetAsync(d.wf_flag, 0, div_up(np, 256), c->stream));
    // bonds and their per-particle lists (by user index, in bond order)
    if (nb0 > 0) {
        std::vector<uint32_t> ptr(np + 1, 0), list;
        for (size_t b = 0; b < nb0; ++b) {
            const uint32_t x = h->bonds[2 * b], y = h->bonds[2 * b + 1];
            if (y >= np) return fail(c, SPH_ERR_BAD_INPUT, "bond partner index out of range");
            if (x < np) ptr[x + 1]++;
            ptr[y + 1]++;
        }
        for (size_t i = 0; i < np; ++i) ptr[i + 1] += ptr[i];
        list.resize(ptr[np]);
        std::vector<uint32_t> fill(ptr.begin(), ptr.end() - 1);
        for (size_t b = 0; b < nb0; ++b) {
            const uint32_t x = h->bonds[2 * b], y = h->bonds[2 * b + 1];
            if (x < np) list[fill[x]++] = (uint32_t)(b << 1);
            list[fill[y]++] = (uint32_t)((b << 1) | 1u);
        }
        CK(cudaMemcpyAsync(d.bond_ptr, ptr.data(), (np + 1) * 4, cudaMemcpyHostToDevice, c->stream));
        if (!list.empty())
            CK(cudaMemcpyAsync(d.bond_list, list.data(), list.size() * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(d.bonds, h->bonds, nb0 * 8, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(d.bonds_delta, h->bonds_delta, nb0 * 32, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(d.bonds_omega, h->bonds_omega, nb0 * 32, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));   // the CSR built above goes out of scope
    }
    CK(cudaMemsetAsync(d.status, 0, 4, c->stream));
    const uint32_t one = 1;
    CK(cudaMemcpyAsync(d.rebuild, &one, 4, cudaMemcpyHostToDevice, c->stream));
    c->sticky = SPH_OK;
    c->err.clear();
    c->t_host = h->t_current;
    c->steps = 0;
    // cell list of the initial positions, then storage in cell order
    launch_cell_init(d, c->np_all, A, c->stream);
    CK(cudaGetLastError());
    int rc = do_relayout(c, c->stream);
    if (rc != SPH_OK) return rc;
    c->uploaded = true;
    // the step graphs carry the force kernel's constants, which the upload
    // may have changed (the skin): capture them here rather than in the
    // first sph_step
    if (!c->batched && (rc = ensure_graphs(c)) != SPH_OK) return rc;
    return sync_status(c);
}

static int step_plain(sph_ctx *c, uint64_t nsteps, void *stream);
static int save_ckpt(sph_ctx *c, sph_ctx::Ckpt &k);

int sph_step(sph_ctx *c, uint64_t nsteps, void *stream)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_step before sph_upload");
    if (!c->diff) return step_plain(c, nsteps, stream);
    // differentiable mode: a checkpoint at every multiple of ckpt_every steps
    if (c->sticky != SPH_OK) return c->sticky;
    CK(cudaSetDevice(c->device));
    const uint64_t K = c->ckpt_every;
    uint64_t left = nsteps;
    while (left > 0) {
        if (c->diff_steps % K == 0 && c->diff_steps / K == c->ckpts.size()) {
            // the copy runs on the context's stream: after the caller's
            // steps so far, and before the caller's next ones
            cudaStream_t us = stream ? static_cast<cudaStream_t>(stream) : c->stream;
            if (!c->ckpt_ev) CK(cudaEventCreateWithFlags(&c->ckpt_ev, cudaEventDisableTiming));
            if (us != c->stream) {
                CK(cudaEventRecord(c->ckpt_ev, us));
                CK(cudaStreamWaitEvent(c->stream, c->ckpt_ev, 0));
            }
            sph_ctx::Ckpt k{};
            const int rc = save_ckpt(c, k);
            if (rc != SPH_OK) return rc;
            c->ckpts.push_back(k);
            if (us != c->stream) {
                CK(cudaEventRecord(c->ckpt_ev, c->stream));
                CK(cudaStreamWaitEvent(us, c->ckpt_ev, 0));
            }
        }
        const uint64_t chunk = std::min<uint64_t>(left, K - c->diff_steps % K);
        const int rc = step_plain(c, chunk, stream);
        if (rc != SPH_OK) return rc;
        left -= chunk;
        c->diff_steps += chunk;
    }
    return SPH_OK;
}

static int step_plain(sph_ctx *c, uint64_t nsteps, void *stream)
{
    if (c->sticky != SPH_OK) return c->sticky;
    if (nsteps == 0) return SPH_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    int rc;
    if (c->profile) {
        for (uint64_t i = 0; i < nsteps; ++i) {
            if (c->relayout_every > 0 && c->since_relayout >= (uint64_t)c->relayout_every)
                if ((rc = do_relayout(c, st)) != SPH_OK) return rc;
            if ((rc = profiled_step(c, c->a, i + 1 == nsteps, st)) != SPH_OK) return rc;
            c->a ^= 1;
            c->since_relayout++;
            c->steps++;
            c->t_host += c->hp.dt;
        }
        return SPH_OK;
    }
    rc = ensure_graphs(c);
    if (rc != SPH_OK) return rc;
    const uint64_t K = (uint64_t)c->graph_steps;
    uint64_t i = 0;
    while (i < nsteps) {
        if (c->relayout_every > 0 && c->since_relayout >= (uint64_t)c->relayout_every) {
            if ((rc = do_relayout(c, st)) != SPH_OK) return rc;
        }
        uint64_t room = nsteps - i;
        if (c->relayout_every > 0) {
            const uint64_t left = (uint64_t)c->relayout_every - c->since_relayout;
            if (left < room) room = left;
        }
        const bool last_chunk = (i + room == nsteps);
        // multi-step graphs while more than one graph's worth remains
        while (room > K || (room == K && !last_chunk)) {
            CK(cudaGraphLaunch(c->g_multi[c->a], st));
            c->a ^= (int)(K & 1u);
            room -= K; i += K; c->since_relayout += K; c->steps += K;
            for (uint64_t k = 0; k < K; ++k) c->t_host += c->hp.dt;
        }
        while (room > 0) {
            const int w = (room == 1 && last_chunk) ? 1 : 0;
            CK(cudaGraphLaunch(c->g_single[c->a][w], st));
            c->a ^= 1;
            room -= 1; i += 1; c->since_relayout += 1; c->steps += 1;
            c->t_host += c->hp.dt;
        }
    }
    return SPH_OK;
}

int sph_sync(sph_ctx *c)
{
    if (!c) return SPH_ERR_BAD_INPUT;
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    if (c->sticky != SPH_OK) return c->sticky;
    return sync_status(c);
}

int sph_download(sph_ctx *c, sph_host_state *h)
{
    if (!c || !h || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_download: bad arguments");
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    const Params &P = c->hp;
    const uint32_t np = c->np_all;
    Dev &d = c->d;
    const int A = c->a;
    const unsigned int grid = div_up(np, 256);
    double4 *t4 = static_cast<double4 *>(c->scratch);
    auto get4 = [&](const double4 *src, double *dst) -> int {
        if (!dst) return SPH_OK;
        k_to_user<double4><<<grid, 256, 0, c->stream>>>(src, t4, d.sidx, np);
        CK(cudaMemcpyAsync(dst, t4, (size_t)np * 32, cudaMemcpyDeviceToHost, c->stream));
        return SPH_OK;
    };
    int rc;
    auto get3 = [&](const P3 *src, int lane, double *dst) -> int {
        if (!dst) return SPH_OK;
        k_p3_to_user<<<grid, 256, 0, c->stream>>>(src, d.w_user, lane, t4, d.sidx, np);
        CK(cudaMemcpyAsync(dst, t4, (size_t)np * 32, cudaMemcpyDeviceToHost, c->stream));
        return SPH_OK;
    };
    if ((rc = get4(d.xr[A], h->x)) || (rc = get3(d.vel[A], W_VEL, h->vel)) ||
        (rc = get3(d.vel0, W_VEL0, h->vel0)) || (rc = get4(d.acc, h->acc)) ||
        (rc = get4(d.force, h->force)) || (rc = get3(d.angpos, W_ANGPOS, h->angpos)) ||
        (rc = get3(d.angvel[A], W_ANGVEL, h->angvel)) || (rc = get3(d.angvel0, W_ANGVEL0, h->angvel0)) ||
        (rc = get4(d.angacc, h->angacc)) || (rc = get4(d.torque, h->torque)))
        return rc;
    {
        // xysum, and the lanes of esv / edp as the caller's planar arrays,
        // copied straight into them
        double2 *t2 = static_cast<double2 *>(c->scratch);
        double *t1 = static_cast<double *>(c->scratch);
        cudaStream_t st = c->stream;
        if (h->xysum) {
            k_to_user<double2><<<grid, 256, 0, st>>>(d.xysum, t2, d.sidx, np);
            CK(cudaMemcpyAsync(h->xysum, t2, (size_t)np * 16, cudaMemcpyDeviceToHost, st));
        }
        const struct { double *dst; int src; } lanes[] = {
            {h->es, 0}, {h->ev, 1}, {h->es_dot, 2}, {h->ev_dot, 3}, {h->p, 4}};
        for (const auto &l : lanes) {
            if (!l.dst) continue;
            switch (l.src) {
            case 0: k_lane_to_user<double2, 0><<<grid, 256, 0, st>>>(d.esv, t1, d.sidx, np); break;
            case 1: k_lane_to_user<double2, 1><<<grid, 256, 0, st>>>(d.esv, t1, d.sidx, np); break;
            case 2: k_lane_to_user<double4, 0><<<grid, 256, 0, st>>>(d.edp, t1, d.sidx, np); break;
            case 3: k_lane_to_user<double4, 1><<<grid, 256, 0, st>>>(d.edp, t1, d.sidx, np); break;
            default: k_lane_to_user<double4, 2><<<grid, 256, 0, st>>>(d.edp, t1, d.sidx, np); break;
            }
            CK(cudaMemcpyAsync(l.dst, t1, (size_t)np * 8, cudaMemcpyDeviceToHost, st));
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
    }
    if (h->contacts || h->distmod || h->delta_t) {
        rc = sph_get_contacts(c, h->contacts, h->distmod, h->delta_t);
        if (rc != SPH_OK) return rc;
    }
    if (P.nb0 > 0) {
        if (h->bonds) CK(cudaMemcpyAsync(h->bonds, d.bonds, (size_t)P.nb0 * 8, cudaMemcpyDeviceToHost, c->stream));
        if (h->bonds_delta) CK(cudaMemcpyAsync(h->bonds_delta, d.bonds_delta, (size_t)P.nb0 * 32, cudaMemcpyDeviceToHost, c->stream));
        if (h->bonds_omega) CK(cudaMemcpyAsync(h->bonds_omega, d.bonds_omega, (size_t)P.nb0 * 32, cudaMemcpyDeviceToHost, c->stream));
    }
    Walls W{};
    CK(cudaMemcpyAsync(&W, d.walls, sizeof(W), cudaMemcpyDeviceToHost, c->stream));
    for (uint32_t k = 0; k < P.nw; ++k) {
        if (h->walls_nx) memcpy(&h->walls_nx[4 * k], &W.nx[k], 32);
        if (h->walls_mvfd) memcpy(&h->walls_mvfd[4 * k], &W.mvfd[k], 32);
        if (h->walls_vel0) h->walls_vel0[k] = W.vel0[k];
    }
    h->t_current = c->t_host;
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    return SPH_OK;
}

int sph_get_contacts(sph_ctx *c, uint32_t *contacts, double *distmod, double *delta_t)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_get_contacts before upload");
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    const uint32_t np = c->np_all;
    const size_t n = (size_t)np * NC;
    uint32_t *dc = nullptr;
    double4 *ddm = nullptr, *ddt = nullptr;
    CK(cudaMallocAsync(&dc, n * 4, c->stream));
    CK(cudaMallocAsync(&ddm, n * 32, c->stream));
    CK(cudaMallocAsync(&ddt, n * 32, c->stream));
    k_rows_to_user<<<div_up(n, 256), 256, 0, c->stream>>>(c->d, dc, ddm, ddt, c->a);
    if (contacts) CK(cudaMemcpyAsync(contacts, dc, n * 4, cudaMemcpyDeviceToHost, c->stream));
    if (distmod) CK(cudaMemcpyAsync(distmod, ddm, n * 32, cudaMemcpyDeviceToHost, c->stream));
    if (delta_t) CK(cudaMemcpyAsync(delta_t, ddt, n * 32, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(dc, c->stream));
    CK(cudaFreeAsync(ddm, c->stream));
    CK(cudaFreeAsync(ddt, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SPH_OK;
}

int sph_get_cells(sph_ctx *c, uint32_t *cell_sorted, uint32_t *perm, uint32_t *cell_start,
                  uint32_t *cell_end)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_get_cells before upload");
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    const uint32_t np = c->np_all, nc = c->ncells_all;
    uint32_t *b = nullptr;
    const size_t words = (size_t)np * 2 + (size_t)nc * 2;
    CK(cudaMallocAsync(&b, words * 4, c->stream));
    uint32_t *cs = b, *pm = b + np, *st = b + 2 * (size_t)np, *en = st + nc;
    const unsigned int n = (np > nc + 1 ? np : nc + 1);
    k_cells_out<<<div_up(n, 256), 256, 0, c->stream>>>(c->d, cs, pm, st, en);
    if (cell_sorted) CK(cudaMemcpyAsync(cell_sorted, cs, (size_t)np * 4, cudaMemcpyDeviceToHost, c->stream));
    if (perm) CK(cudaMemcpyAsync(perm, pm, (size_t)np * 4, cudaMemcpyDeviceToHost, c->stream));
    if (cell_start) CK(cudaMemcpyAsync(cell_start, st, (size_t)nc * 4, cudaMemcpyDeviceToHost, c->stream));
    if (cell_end) CK(cudaMemcpyAsync(cell_end, en, (size_t)nc * 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaFreeAsync(b, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SPH_OK;
}

int sph_get_wall_forces(sph_ctx *c, double *wall0_force)
{
    if (!c || !c->uploaded || !wall0_force) return fail(c, SPH_ERR_BAD_INPUT, "bad arguments");
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpyAsync(wall0_force, c->d.wf_pp, (size_t)c->np_all * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    return SPH_OK;
}

int sph_get_stats(sph_ctx *c, sph_stats *out)
{
    if (!c || !out) return SPH_ERR_BAD_INPUT;
    CK(cudaSetDevice(c->device));
    memset(out, 0, sizeof(*out));
    if (c->uploaded) {
        unsigned long long *cnt = nullptr;
        CK(cudaMallocAsync(&cnt, 8, c->stream));
        CK(cudaMemsetAsync(cnt, 0, 8, c->stream));
        k_count_contacts<<<592, 256, 0, c->stream>>>(c->d.cmask, c->np_all, cnt);
        unsigned long long v = 0;
        CK(cudaMemcpyAsync(&v, cnt, 8, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaFreeAsync(cnt, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        out->active_contacts = v;
    }
    if (c->uploaded) {
        Verlet V{};
        CK(cudaMemcpyAsync(&V, c->d.vs, sizeof(V), cudaMemcpyDeviceToHost, c->stream));
        out->cell_rebuilds = V.rebuilds;
    }
    out->steps = c->steps;
    out->relayouts = c->relayouts;
    out->device_bytes = c->device_bytes + c->diff_bytes +
                        (c->ckpts.size() + c->ckpt_pool.size()) * c->ckpt_bytes;
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    return SPH_OK;
}

int sph_get_profile(sph_ctx *c, double *ms, uint64_t *steps, int reset)
{
    if (!c) return SPH_ERR_BAD_INPUT;
    for (int k = 0; k < SPH_NPHASES; ++k) {
        if (ms) ms[k] = c->prof_ms[k];
        if (reset) c->prof_ms[k] = 0.0;
    }
    if (steps) *steps = c->prof_steps;
    if (reset) c->prof_steps = 0;
    return SPH_OK;
}

int sph_relayout(sph_ctx *c)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_relayout before upload");
    CK(cudaSetDevice(c->device));
    int rc = do_relayout(c, c->stream);
    if (rc != SPH_OK) return rc;
    return sync_status(c);
}

// ---- differentiable mode ---------------------------------------------------

// The arrays a checkpoint holds, in order: the state a step reads and
// carries (buffer `a` of the double-buffered kinematics) and the contact
// slots with their history.  Cell lists and Verlet lists are rebuilt on
// restore; results do not depend on them.
static std::vector<std::pair<void *, size_t>> ckpt_fields(sph_ctx *c, int a)
{
    Dev &d = c->d;
    const size_t np = c->np_all;
    return {{d.xr[a], np * 32},       {d.vel[a], np * 24},  {d.angvel[a], np * 24},
            {d.vel0, np * 24},        {d.angvel0, np * 24}, {d.angpos, np * 24},
            {d.xysum, np * 16},       {d.esv, np * 16},     {d.contacts, tiled_size(np, NC) * 4},
            {d.dmc, np * 16},         {d.cmask, np * 4},
            {d.delta_t, tiled_size(np, NC) * sizeof(P3)}};
}

static int save_ckpt(sph_ctx *c, sph_ctx::Ckpt &k)
{
    k.a = c->a;
    k.t_host = c->t_host;
    size_t bytes = 0;
    for (auto &f : ckpt_fields(c, c->a)) bytes += f.second;
    k.buf = nullptr;
    if (c->ckpt_bytes != bytes) {
        for (char *b : c->ckpt_pool) cudaFree(b);
        c->ckpt_pool.clear();
        c->ckpt_bytes = bytes;
    }
    if (!c->ckpt_pool.empty()) {
        k.buf = c->ckpt_pool.back();
        c->ckpt_pool.pop_back();
    } else {
        // fully overwritten below, so no clearing
        CK(cudaMalloc(&k.buf, bytes));
    }
    size_t off = 0;
    for (auto &f : ckpt_fields(c, c->a)) {
        CK(cudaMemcpyAsync(k.buf + off, f.first, f.second, cudaMemcpyDeviceToDevice, c->stream));
        off += f.second;
    }
    return SPH_OK;
}

static void ckpt_release(sph_ctx *c, char *buf)
{
    if (buf) c->ckpt_pool.push_back(buf);
}

static int restore_ckpt(sph_ctx *c, const sph_ctx::Ckpt &k)
{
    c->a = k.a;
    c->t_host = k.t_host;
    size_t off = 0;
    for (auto &f : ckpt_fields(c, k.a)) {
        CK(cudaMemcpyAsync(f.first, k.buf + off, f.second, cudaMemcpyDeviceToDevice, c->stream));
        off += f.second;
    }
    Dev &d = c->d;
    launch_cell_init(d, c->np_all, k.a, c->stream);
    CK(cudaMemsetAsync(d.dirty, 0, ((size_t)c->ncells_all + 1) * sizeof(uint32_t), c->stream));
    CK(cudaMemsetAsync(d.cflag, 1, div_up(c->np_all, 32), c->stream));
    CK(cudaMemsetAsync(d.settled, 0, c->np_all, c->stream));
    // stream-ordered: the host enqueues the next work without waiting
    launch_epoch_reset(d, c->stream);
    CK(cudaGetLastError());
    return SPH_OK;
}

// One segment of the backward pass as a graph: the `len` steps re-run from
// the restored checkpoint (buffer a) recording tape rows 0 .. len-1, then the
// reverse of each step, last first.
static int capture_segment(sph_ctx *c, int len, int a, cudaGraphExec_t *out)
{
    Dev &d = c->d;
    const uint32_t np = c->np_all;
    cudaStream_t st = c->stream;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = SPH_OK;
    int aa = a;
    for (int j = 0; j < len && rc == SPH_OK; ++j) {
        if (c->cond_rebuild) rc = capture_rebuild_conditional(c, aa, st);
        else launch_rebuild(d, np, c->ncells_all, aa, st);
        launch_topo(d, np, false, aa, st);
        launch_force_tape(d, np, aa, j, st);
        launch_walls(d, np, 0, st);
        aa ^= 1;
    }
    for (int j = len - 1; j >= 0 && rc == SPH_OK; --j) launch_rev_step(d, c->adj, np, j, st);
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != SPH_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(c, SPH_ERR_CUDA, std::string("segment capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return fail(c, SPH_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    return SPH_OK;
}

static void free_diff(sph_ctx *c)
{
    for (auto &kv : c->diff_graphs)
        if (kv.second) cudaGraphExecDestroy(kv.second);
    c->diff_graphs.clear();
    for (void *p : c->diff_allocs) cudaFree(p);
    c->diff_allocs.clear();
    c->bwd_scratch = nullptr;
    c->diff_bytes = 0;
    for (auto &k : c->ckpts) ckpt_release(c, k.buf);
    c->ckpts.clear();
    c->adj = AdjDev{};
    Dev &d = c->d;
    d.mu_p = nullptr;
    d.tp_x = d.tp_v = d.tp_w = nullptr;
    d.tp_dt0 = nullptr;
    d.tp_mask = d.tp_partner = nullptr;
    d.tp_dmc = nullptr;
}

int sph_diff_begin(sph_ctx *c, const double *mu, uint32_t checkpoint_every)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_diff_begin before sph_upload");
    if (c->diff) return fail(c, SPH_ERR_BAD_INPUT, "sph_diff_begin: already in differentiable mode");
    const Params &P = c->hp;
    if (c->batched || P.contactmodel != 2 || P.nw != 0 || P.nb0 != 0 || c->darcy_on)
        return fail(c, SPH_ERR_BAD_INPUT,
                    "the differentiable step takes one scene with contact model 2, no dynamic "
                    "walls, no bonds and no Darcy flow");
    if (checkpoint_every == 0) return fail(c, SPH_ERR_BAD_INPUT, "checkpoint_every must be >= 1");
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    const size_t np = c->np_all, K = checkpoint_every;
    Dev &d = c->d;
    AdjDev &A = c->adj;
    std::vector<void *> *own = &c->diff_allocs;
    int rc = SPH_OK;
#define ALD(ptr, n) if ((rc = dalloc(c, &(ptr), (n), own)) != SPH_OK) { free_diff(c); return rc; }
    ALD(d.mu_p, np);
    ALD(d.tp_x, K * np); ALD(d.tp_v, K * np); ALD(d.tp_w, K * np);
    ALD(d.tp_mask, K * np); ALD(d.tp_dmc, K * np);
    ALD(d.tp_partner, K * tiled_size(np, NC)); ALD(d.tp_dt0, K * tiled_size(np, NC));
    ALD(A.xb, np); ALD(A.vb, np); ALD(A.wb, np); ALD(A.v0b, np); ALD(A.w0b, np);
    ALD(A.Fb, np); ALD(A.Tb, np); ALD(A.dtb, tiled_size(np, NC)); ALD(A.mub, np); ALD(A.theta_b, 3);
    ALD(A.dtb_mask, np);
    double *tmp = nullptr;
    ALD(tmp, np);
#undef ALD
    if (mu) CK(cudaMemcpyAsync(tmp, mu, np * 8, cudaMemcpyHostToDevice, c->stream));
    launch_user_to_storage1(mu ? tmp : nullptr, d.mu_p, d.uid, P.mu_s, (uint32_t)np, c->stream);
    CK(cudaStreamSynchronize(c->stream));
    // kernels and graphs take Dev by value: capture again with the new arrays
    drop_graphs(c);
    c->relayout_saved = c->relayout_every;
    c->relayout_every = 0;   // the tape and checkpoints are storage-indexed
    c->diff = true;
    c->ckpt_every = checkpoint_every;
    c->diff_steps = 0;
    sph_ctx::Ckpt k{};
    if ((rc = save_ckpt(c, k)) != SPH_OK) return rc;
    c->ckpts.push_back(k);
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    return SPH_OK;
}

int sph_diff_backward(sph_ctx *c, const double *x_bar, const double *v_bar, double *grad_params,
                      double *grad_mu, double *x0_bar, double *v0_bar)
{
    if (!c || !c->diff) return fail(c, SPH_ERR_BAD_INPUT, "sph_diff_backward outside differentiable mode");
    if (c->sticky != SPH_OK) return c->sticky;
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    const uint32_t np = c->np_all;
    const uint64_t N = c->diff_steps, K = c->ckpt_every;
    Dev &d = c->d;
    AdjDev &A = c->adj;
    cudaStream_t st = c->stream;
    // the state after the forward, put back at the end
    sph_ctx::Ckpt fin{};
    int rc = save_ckpt(c, fin);
    if (rc != SPH_OK) return rc;
    // seeds: dL/dx and dL/dv of the current state; the scratch stays for the
    // rest of the differentiable session
    if (!c->bwd_scratch && (rc = dalloc(c, &c->bwd_scratch, 13 * (size_t)np, &c->diff_allocs)))
        return rc;
    double *hx = c->bwd_scratch;
    double *out = c->bwd_scratch + 6 * (size_t)np;
    {
        if (x_bar) CK(cudaMemcpyAsync(hx, x_bar, (size_t)np * 24, cudaMemcpyHostToDevice, c->stream));
        if (v_bar) CK(cudaMemcpyAsync(hx + 3 * (size_t)np, v_bar, (size_t)np * 24, cudaMemcpyHostToDevice, c->stream));
        launch_user_to_storage3(x_bar ? hx : nullptr, A.xb, d.uid, np, st);
        launch_user_to_storage3(v_bar ? hx + 3 * (size_t)np : nullptr, A.vb, d.uid, np, st);
    }
    for (double4 *p : {A.wb, A.v0b, A.w0b}) CK(cudaMemsetAsync(p, 0, (size_t)np * 32, st));
    CK(cudaMemsetAsync(A.dtb, 0, tiled_size(np, NC) * sizeof(P3), st));
    CK(cudaMemsetAsync(A.dtb_mask, 0, (size_t)np * 4, st));
    CK(cudaMemsetAsync(A.mub, 0, (size_t)np * 8, st));
    CK(cudaMemsetAsync(A.theta_b, 0, 24, st));
    const uint64_t nseg = (N + K - 1) / K;
    for (uint64_t seg = nseg; seg-- > 0;) {
        // adjoints survive the restore: they live apart from the state
        if ((rc = restore_ckpt(c, c->ckpts[seg])) != SPH_OK) return rc;
        const int len = (int)std::min<uint64_t>(K, N - seg * K);
        cudaGraphExec_t &gx = c->diff_graphs[{len, c->a}];
        if (!gx && (rc = capture_segment(c, len, c->a, &gx)) != SPH_OK) return rc;
        CK(cudaGraphLaunch(gx, st));
    }
    if ((rc = restore_ckpt(c, fin)) != SPH_OK) return rc;
    if ((rc = sync_status(c)) != SPH_OK) return rc;
    // results in the caller's order
    launch_storage_to_user1(A.mub, out, d.sidx, np, st);
    launch_storage_to_user3(A.xb, nullptr, out + np, d.sidx, np, st);
    launch_storage_to_user3(A.vb, A.v0b, out + 4 * (size_t)np, d.sidx, np, st);
    CK(cudaStreamSynchronize(st));
    if (grad_params) CK(cudaMemcpyAsync(grad_params, A.theta_b, 24, cudaMemcpyDeviceToHost, c->stream));
    if (grad_mu) CK(cudaMemcpyAsync(grad_mu, out, (size_t)np * 8, cudaMemcpyDeviceToHost, c->stream));
    if (x0_bar) CK(cudaMemcpyAsync(x0_bar, out + np, (size_t)np * 24, cudaMemcpyDeviceToHost, c->stream));
    if (v0_bar) CK(cudaMemcpyAsync(v0_bar, out + 4 * (size_t)np, (size_t)np * 24, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    ckpt_release(c, fin.buf);   // the final-state copy goes back to the pool
    return SPH_OK;
}

int sph_diff_end(sph_ctx *c)
{
    if (!c) return SPH_ERR_BAD_INPUT;
    if (!c->diff) return SPH_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    free_diff(c);
    drop_graphs(c);
    CK(cudaMemsetAsync(c->d.cflag, 1, div_up(c->np_all, 32), c->stream));
    CK(cudaMemsetAsync(c->d.settled, 0, c->np_all, c->stream));
    c->diff = false;
    c->relayout_every = c->relayout_saved;
    return SPH_OK;
}

int sph_darcy_upload(sph_ctx *c, double nu, const sph_darcy_state *h)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_darcy_upload before sph_upload");
    if (c->batched || c->diff)
        return fail(c, SPH_ERR_BAD_INPUT, "Darcy flow needs a plain (not batched or differentiable) context");
    if (!(nu > 0.0)) return fail(c, SPH_ERR_BAD_INPUT, "Darcy flow needs a dynamic viscosity nu > 0");
    if (!h || !h->H || !h->H_new || !h->V || !h->dH || !h->K || !h->T || !h->Ss || !h->W || !h->phi ||
        !h->dphi)
        return fail(c, SPH_ERR_BAD_INPUT, "sph_darcy_upload: missing array");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    const size_t n = (size_t)(c->hp.num[0] + 2) * (c->hp.num[1] + 2) * (c->hp.num[2] + 2);
    DarcyDev &f = c->darcy;
    int rc;
    if (!f.first) {
        if ((rc = dalloc(c, &f.H[0], n)) || (rc = dalloc(c, &f.H[1], n)) ||
            (rc = dalloc(c, &f.V, 3 * n)) || (rc = dalloc(c, &f.dH, 3 * n)) ||
            (rc = dalloc(c, &f.K, n)) || (rc = dalloc(c, &f.T, 3 * n)) ||
            (rc = dalloc(c, &f.Ss, n)) || (rc = dalloc(c, &f.W, n)) ||
            (rc = dalloc(c, &f.phi, n)) || (rc = dalloc(c, &f.dphi, n)) ||
            (rc = dalloc(c, &f.first, 1)))
            return rc;
    }
    // the uploaded pressure is the current one for the context's parity
    c->dflip = c->a;
    const std::pair<double *, const double *> one[] = {
        {f.H[0], h->H}, {f.H[1], h->H_new}, {f.K, h->K}, {f.Ss, h->Ss},
        {f.W, h->W},    {f.phi, h->phi},    {f.dphi, h->dphi}};
    for (const auto &p : one) CK(cudaMemcpyAsync(p.first, p.second, n * 8, cudaMemcpyHostToDevice, c->stream));
    const std::pair<double *, const double *> three[] = {{f.V, h->V}, {f.dH, h->dH}, {f.T, h->T}};
    for (const auto &p : three) CK(cudaMemcpyAsync(p.first, p.second, 3 * n * 8, cudaMemcpyHostToDevice, c->stream));
    const uint32_t one_u = 1u;
    CK(cudaMemcpyAsync(f.first, &one_u, 4, cudaMemcpyHostToDevice, c->stream));
    f.nu = nu;
    // src/device.cu:673-678
    const double r_bar2 = c->mean_radius * 2.0;
    f.d_factor = r_bar2 * r_bar2 / 180.0 * 1.0e-6;
    if (!c->darcy_stream) {
        CK(cudaStreamCreateWithFlags(&c->darcy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->darcy_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->darcy_join, cudaEventDisableTiming));
    }
    c->darcy_on = true;
    drop_graphs(c);   // the step graphs gain the Darcy kernels
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    return SPH_OK;
}

int sph_darcy_download(sph_ctx *c, sph_darcy_state *h)
{
    if (!c || !c->darcy_on) return fail(c, SPH_ERR_BAD_INPUT, "sph_darcy_download without sph_darcy_upload");
    if (!h) return fail(c, SPH_ERR_BAD_INPUT, "sph_darcy_download: null state");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    const size_t n = (size_t)(c->hp.num[0] + 2) * (c->hp.num[1] + 2) * (c->hp.num[2] + 2);
    const DarcyDev &f = c->darcy;
    const int hs = c->a ^ c->dflip;
    const std::pair<double *, const double *> one[] = {
        {h->H, f.H[hs]}, {h->H_new, f.H[hs ^ 1]}, {h->K, f.K},      {h->Ss, f.Ss},
        {h->W, f.W},     {h->phi, f.phi},         {h->dphi, f.dphi}};
    for (const auto &p : one)
        if (p.first) CK(cudaMemcpyAsync(p.first, p.second, n * 8, cudaMemcpyDeviceToHost, c->stream));
    const std::pair<double *, const double *> three[] = {{h->V, f.V}, {h->dH, f.dH}, {h->T, f.T}};
    for (const auto &p : three)
        if (p.first) CK(cudaMemcpyAsync(p.first, p.second, 3 * n * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));   // the caller's arrays are complete
    return SPH_OK;
}

int sph_render(sph_ctx *c, const sph_render_opts *o, uint8_t *rgba)
{
    if (!c || !c->uploaded) return fail(c, SPH_ERR_BAD_INPUT, "sph_render before sph_upload");
    if (c->batched) return fail(c, SPH_ERR_BAD_INPUT, "sph_render takes a single-scene context");
    if (!o || !rgba || o->method < 0 || o->method > 5 || o->width == 0 || o->height == 0)
        return fail(c, SPH_ERR_BAD_INPUT, "sph_render: bad options");
    const uint64_t pixels = (uint64_t)o->width * o->height;
    if (pixels >= (1ull << 24))
        return fail(c, SPH_ERR_TOO_LARGE, "sph_render: width * height must stay below 2^24");
    CK(cudaSetDevice(c->device));
    const size_t np = c->np_all;
    const size_t need = 32 + pixels * 8 + pixels * 4 + np * 8 + (size_t)o->width * 24;
    if (c->rt_bytes < need) {
        if (c->rt_buf) cudaFree(c->rt_buf);
        c->rt_buf = nullptr;
        c->rt_bytes = 0;
        CK(cudaMalloc(&c->rt_buf, need));
        c->rt_bytes = need;
    }
    char *base = static_cast<char *>(c->rt_buf);
    auto *mx = reinterpret_cast<unsigned long long *>(base);
    auto *keys = reinterpret_cast<unsigned long long *>(base + 32);
    auto *img = reinterpret_cast<uchar4 *>(base + 32 + pixels * 8);
    auto *values = reinterpret_cast<double *>(base + 32 + pixels * 12);
    auto *rays = reinterpret_cast<float *>(base + 32 + pixels * 12 + np * 8);
    cudaStream_t st = c->stream;
    // DEM::maxPos on the device, then the camera on the host
    CK(cudaMemsetAsync(mx, 0, 24, st));
    launch_maxpos(c->d, c->np_all, c->a, mx, st);
    unsigned long long mxh[3];
    CK(cudaMemcpyAsync(mxh, mx, 24, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double maxpos[3];
    for (int k = 0; k < 3; ++k) memcpy(&maxpos[k], &mxh[k], 8);
    CK(cudaMemsetAsync(keys, 0xff, pixels * 8, st));
    render_image(c->d, c->np_all, c->a, c->hp.L, maxpos, *o, values, keys, img, rays, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rgba, img, pixels * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SPH_OK;
}

int sph_destroy(sph_ctx *c)
{
    if (!c) return SPH_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    for (auto e : c->ev) cudaEventDestroy(e);
    free_diff(c);
    for (char *b : c->ckpt_pool) cudaFree(b);
    if (c->rt_buf) cudaFree(c->rt_buf);
    if (c->ckpt_ev) cudaEventDestroy(c->ckpt_ev);
    if (c->darcy_fork) cudaEventDestroy(c->darcy_fork);
    if (c->darcy_join) cudaEventDestroy(c->darcy_join);
    if (c->darcy_stream) cudaStreamDestroy(c->darcy_stream);
    if (c->wall_fork) cudaEventDestroy(c->wall_fork);
    if (c->wall_join) cudaEventDestroy(c->wall_join);
    if (c->wall_stream) cudaStreamDestroy(c->wall_stream);
    for (void *p : c->allocs) cudaFree(p);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->side) cudaStreamDestroy(c->side);
    delete c;
    return SPH_OK;
}

}  // extern "C"
