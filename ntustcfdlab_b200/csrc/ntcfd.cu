// ntcfd.cu -- device context and C-ABI of the B200 projection-method step.
//
// One context = one grid resident in device memory + one CUDA stream + one
// instantiated CUDA graph holding a whole time step (main.f90:209-259).  The
// SOR loop of gauss_seidel (GS.f90:11) runs on the device as a nested pair
// of conditional WHILE nodes (defect-correction cycles around red-black
// sweeps), so a step needs no host round trip; ntcfd_step(n) launches the
// graph n times and copies back one small record per step.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ntcfd.h"
#include "k_adjoint.cuh"
#include "k_mask.cuh"
#include "k_predictor.cuh"
#include "k_predictor32.cuh"
#include "k_schemes.cuh"
#include "k_pressure.cuh"
#include "k_project.cuh"
#include "k_resident.cuh"
#include "ntcfd_common.cuh"

using namespace ntcfd;

namespace {

constexpr int kProjKc = 8;      // planes per column chunk in K4
constexpr int kSweepNT = 256;    // threads per CTA of a streaming half-sweep
constexpr int kSweepBx = 64;     // column form: threads per row, rows per CTA, planes per thread
constexpr int kSweepBy = 4;
constexpr int kSweepKpt = 4;
constexpr int kResNT = 512;      // threads per CTA of the resident SOR kernel
constexpr int kMixedCycle = 8;   // default FP32 sweeps per defect-correction cycle (mixed_cycle = 0)
constexpr int kAdjQueued = 16;   // loop bodies an adjoint solve queues per host round trip (streaming)
const double kZeroZeta = 0.0;
const int kOne = 1;

// The streaming half-sweep of a precision.  FP64 moves 40 B per cell and runs
// closest to the HBM bandwidth in the column form (four planes per thread,
// 36 loads in flight); FP32 is instruction-bound in that form and faster with
// one warp per row.  Both do the same arithmetic per cell.
template <class Tc>
struct Sweep;
template <>
struct Sweep<double> {
    static constexpr auto fn = k_sweep_cols<double, kSweepBx * kSweepBy, kSweepKpt>;
    static dim3 block() { return dim3(kSweepBx, kSweepBy, 1); }
    static dim3 grid(const Geom& g, int) {
        const int half = (g.nx + 1) / 2;
        return dim3((half + kSweepBx - 1) / kSweepBx, (g.ny + kSweepBy - 1) / kSweepBy,
                    (g.nz + kSweepKpt - 1) / kSweepKpt);
    }
};
// The row sweep (FP32) takes a cycle's first sweep with e read as zero; the
// column sweep (FP64) runs after k_clear_e.
template <class Tc>
constexpr bool kRowSweep = sizeof(Tc) == 4;

template <>
struct Sweep<float> {
    static constexpr auto fn = k_sweep_rows<float, kSweepNT>;
    static dim3 block() { return dim3(kSweepNT); }
    static dim3 grid(const Geom& g, int resident) { return sweep_grid(g, kSweepNT, resident); }
};

struct DevTabs {
    // one allocation per precision; every table has n+5 entries (index -2..n+2)
    void* buf = nullptr;
};

}  // namespace

struct ntcfd_ctx {
    ntcfd_params prm{};
    std::string err;
    cudaStream_t stream = nullptr;
    Geom g{};
    size_t nat_elems = 0, spl_elems = 0;
    double *u = nullptr, *v = nullptr, *w = nullptr, *p = nullptr;
    double *us = nullptr, *vs = nullptr, *ws = nullptr, *b = nullptr;
    double *eta = nullptr, *nut = nullptr;
    double* fb = nullptr;                   // body force fu, fv, fw (3 natural arrays), null when unset
    void *eR = nullptr, *eB = nullptr, *dR = nullptr, *dB = nullptr;
    void *rdR = nullptr, *rdB = nullptr;   // 1/diag per colour (sweep precision)
    double* tabd = nullptr;   // double tables
    float* tabf = nullptr;    // float tables
    Tabs<double> tpd{};
    Tabs<float> tpf{};
    SorCoef<double> scd{};
    SorCoef<float> scf{};
    double *partZ = nullptr, *partY = nullptr, *FXz = nullptr, *FYz = nullptr;
    double *FXy = nullptr, *FYy = nullptr;
    unsigned int* fdone = nullptr;         // block counter of k_force_total
    double *faceW = nullptr, *faceE = nullptr, *faceS = nullptr, *faceN = nullptr;
    double *faceB = nullptr, *faceF = nullptr;
    double* outbuf = nullptr;   // pre, uc, vc, wc
    double* stage = nullptr;    // one halo array, contiguous: host <-> device copies of the state
    double *coordY = nullptr, *coordZ = nullptr;  // node coordinates (pre-offset)
    double* coordbuf = nullptr;
    Ctl* ctl = nullptr;
    StepRec* rec = nullptr;
    int rec_cap = 0;
    StepRec* rec_host = nullptr;            // pinned copy of the records of one ntcfd_step call
    int rec_host_cap = 0;
    unsigned long long* slots = nullptr;   // per-sweep max |change| bits
    unsigned long long* divslot = nullptr;
    GridBar* bar = nullptr;                 // grid barrier of the resident SOR kernel
    unsigned long long* ring = nullptr;     // its per-sweep max |change| ring
    Brick brick{};
    bool resident = false;                  // the graph uses the resident SOR kernel
    size_t res_smem = 0;
    int res_grid = 0;
    int sm_count = 0;
    int row_resident = 1;                   // resident blocks of k_sweep_rows (its grid cap)
    int p32_resident = 1;                   // and of k_predictor32 (its waves)
    int defect_resident = 1;                // and of k_defect_rows
    size_t smem_optin = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.0f;
    bool metrics_set = false, coords_set = false;
    bool mask_nonzero = false;              // ETA may be nonzero: the force kernels run
    double* deta_daoa = nullptr;            // ntcfd_build_mask_smooth: dETA_1/dAOA (ny*nz), per radian
    bool smooth_active = false;             // ETA is the smoothed mask that deta_daoa belongs to
    double time = 0.0;
    int nchunk = 0, csweeps = 1, cycle_len = 1;
    std::vector<void*> allocs;
    void* adj_buf = nullptr;                // ntcfd_adjoint workspace, kept between calls
    size_t adj_cap = 0;
    long long istep = 0;                    // steps taken by ntcfd_step since ntcfd_create
    // dynamic angle of attack (ntcfd_set_dynamic_aoa); dyn_start = 0: off
    double dyn_aoa1 = 0.0, dyn_rf = 0.0;
    int dyn_start = 0;
    // its mask on the device (a second step graph: mask kernels, then the step
    // under an IF node that a tie switches off)
    DynMask dyn{};
    void* dyn_buf = nullptr;                // the DynMask arrays
    int dyn_cap = 0;                        // polygon points they hold
    double* dyn_trig = nullptr;             // cos, sin of each step's angle (call-indexed)
    int dyn_trig_cap = 0;
    Ctl* ctl_host = nullptr;                // pinned copy of the control block at the end of a call
    cudaGraph_t graph_dyn = nullptr;
    cudaGraphExec_t exec_dyn = nullptr;
    std::string dyn_graph_err;              // why the device path is off (host path used instead)
    // asynchronous output (ntcfd_output_async)
    cudaStream_t out_stream = nullptr;
    cudaEvent_t out_ready = nullptr, out_done = nullptr;
    double* out_dev = nullptr;              // pre, uc, vc, wc on the device
    double* out_host = nullptr;             // pinned staging for pageable destinations
    double* out_dst[4] = {nullptr, nullptr, nullptr, nullptr};
    bool out_staged[4] = {false, false, false, false};
    size_t out_n = 0;
    bool out_pending = false;
};

namespace {

int fail(ntcfd_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

// The step graphs hold buffer pointers and the mask flag: any change drops them
// and the next ntcfd_step rebuilds.
// A z-slab context: a Back or Front face is shared with a neighbouring slab.
bool is_slab(const ntcfd_ctx* c) {
    return c->prm.bc[NTCFD_BACK][0] == NTCFD_BC_INTERFACE || c->prm.bc[NTCFD_FRONT][0] == NTCFD_BC_INTERFACE;
}

int back_iface(const ntcfd_ctx* c) { return c->prm.bc[NTCFD_BACK][0] == NTCFD_BC_INTERFACE ? 1 : 0; }

void drop_dyn_graph(ntcfd_ctx* c) {
    if (c->exec_dyn) { cudaGraphExecDestroy(c->exec_dyn); c->exec_dyn = nullptr; }
    if (c->graph_dyn) { cudaGraphDestroy(c->graph_dyn); c->graph_dyn = nullptr; }
}

void drop_graphs(ntcfd_ctx* c) {
    if (c->exec) { cudaGraphExecDestroy(c->exec); c->exec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    drop_dyn_graph(c);
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? NTCFD_ENOMEM : NTCFD_ECUDA, \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                        \
    } while (0)

// Every entry point that touches the device selects the context's device
// first: the caller may have another device current on this thread.
#define DEV()                                                                         \
    do {                                                                              \
        if (!ctx || !ctx->stream) return NTCFD_ESTATE;                                \
        CK(cudaSetDevice(ctx->prm.device));                                           \
    } while (0)

template <class T>
int dalloc(ntcfd_ctx* ctx, T** ptr, size_t n) {
    void* q = nullptr;
    CK(cudaMalloc(&q, n * sizeof(T) + 256));
    CK(cudaMemsetAsync(q, 0, n * sizeof(T) + 256, ctx->stream));
    ctx->allocs.push_back(q);
    *ptr = reinterpret_cast<T*>(q);
    return 0;
}

// True when the copy engine reaches p directly: pinned (page-locked or
// registered) host memory, device or managed memory.  Ordinary pageable
// memory reports cudaMemoryTypeUnregistered.
bool dma_reachable(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Stream host function of ntcfd_output_async: moves the staged fields into
// the caller's pageable arrays on the driver's callback thread, so the
// caller's thread keeps issuing steps meanwhile.  It makes no CUDA call.
void CUDART_CB scatter_output(void* arg) {
    auto* ctx = static_cast<ntcfd_ctx*>(arg);
    const size_t n = ctx->out_n;
    for (int q = 0; q < 4; ++q)
        if (ctx->out_staged[q]) std::memcpy(ctx->out_dst[q], ctx->out_host + q * n, n * sizeof(double));
}

// Launch shape of the column-walking kernel k_rhs: 32 x 8 threads
// over (i, j) and enough chunks of k for about two waves of 8 blocks per SM.
dim3 walk_block() { return dim3(kWalkBX, kWalkBY, 1); }
dim3 walk_grid(const Geom& g, int sms) {
    const int bx = (g.nx + kWalkBX - 1) / kWalkBX, by = (g.ny + kWalkBY - 1) / kWalkBY;
    int chunks = (2 * 8 * std::max(sms, 1) + bx * by - 1) / (bx * by);
    chunks = std::max(1, std::min(chunks, g.nz));
    const int kc = (g.nz + chunks - 1) / chunks;
    return dim3(bx, by, (g.nz + kc - 1) / kc);
}

dim3 grid3(const Geom& g, dim3 b) {
    return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y, (g.nz + b.z - 1) / b.z);
}

// Launch shape of the FP32 predictor: 32 x 8 columns, chunks of kc planes;
// the dynamic shared memory holds the chunk's z tables.
dim3 p32_grid(const Geom& g, int kc) {
    return dim3((g.nx + kP32BX - 1) / kP32BX, (g.ny + kP32BY - 1) / kP32BY, (g.nz + kc - 1) / kc);
}
size_t p32_smem(int kc) { return sizeof(float) * 6 * (size_t)(kc + 5); }

// ---- graph construction helpers
template <class Tuple, size_t... I>
void fill_ptrs(Tuple& t, void** p, std::index_sequence<I...>) {
    ((p[I] = (void*)&std::get<I>(t)), ...);
}

template <class... KArgs, class... Args>
cudaError_t add_kernel(cudaGraphNode_t* out, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
                       void (*f)(KArgs...), dim3 grid, dim3 block, Args&&... args) {
    std::tuple<KArgs...> t(std::forward<Args>(args)...);
    void* ptrs[sizeof...(KArgs) > 0 ? sizeof...(KArgs) : 1];
    fill_ptrs(t, ptrs, std::index_sequence_for<KArgs...>{});
    cudaKernelNodeParams kp{};
    kp.func = (void*)f;
    kp.gridDim = grid;
    kp.blockDim = block;
    kp.sharedMemBytes = 0;
    kp.kernelParams = ptrs;
    kp.extra = nullptr;
    return cudaGraphAddKernelNode(out, g, deps.data(), deps.size(), &kp);
}

// A kernel node with dynamic shared memory, optionally cooperative (all CTAs
// co-resident, required by the grid barrier of the resident SOR kernel).
template <class... KArgs, class... Args>
cudaError_t add_kernel_ex(cudaGraphNode_t* out, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
                          void (*f)(KArgs...), dim3 grid, dim3 block, size_t smem, bool cooperative,
                          Args&&... args) {
    std::tuple<KArgs...> t(std::forward<Args>(args)...);
    void* ptrs[sizeof...(KArgs) > 0 ? sizeof...(KArgs) : 1];
    fill_ptrs(t, ptrs, std::index_sequence_for<KArgs...>{});
    cudaKernelNodeParams kp{};
    kp.func = (void*)f;
    kp.gridDim = grid;
    kp.blockDim = block;
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = ptrs;
    kp.extra = nullptr;
    cudaError_t e = cudaGraphAddKernelNode(out, g, deps.data(), deps.size(), &kp);
    if (e != cudaSuccess || !cooperative) return e;
    cudaKernelNodeAttrValue v{};
    v.cooperative = 1;
    return cudaGraphKernelNodeSetAttribute(*out, cudaKernelNodeAttributeCooperative, &v);
}

cudaError_t add_while(cudaGraphNode_t* out, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps,
                      cudaGraphConditionalHandle h, cudaGraph_t* body) {
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaError_t e = cudaGraphAddNode(out, g, deps.data(), deps.size(), &np);
    if (e == cudaSuccess) *body = np.conditional.phGraph_out[0];
    return e;
}

#define GK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(ctx, NTCFD_ECUDA, "graph build: %s: %s (line %d)", #call,        \
                        cudaGetErrorString(e_), __LINE__);                              \
    } while (0)

template <class Tc>
SorCoef<Tc> sor_coef(ntcfd_ctx* ctx);
template <>
SorCoef<double> sor_coef<double>(ntcfd_ctx* ctx) { return ctx->scd; }
template <>
SorCoef<float> sor_coef<float>(ntcfd_ctx* ctx) { return ctx->scf; }

// The resident SOR kernel for a brick plan (d and rd cached or not, row shape).
template <class Tc>
using ResidentFn = void (*)(Geom, SorCoef<Tc>, Brick, double*, const double*, Tc*, Tc*, Tc*, Tc*, const Tc*,
                            const Tc*, Ctl*, GridBar*, double, double, int, int, int, unsigned long long*);
template <class Tc, int MODE>
ResidentFn<Tc> resident_kernel_m(const Brick& b) {
    if (b.cache_d && b.cache_rd) return k_sor_resident<Tc, kResNT, true, true, MODE>;
    if (b.cache_d) return k_sor_resident<Tc, kResNT, true, false, MODE>;
    if (b.cache_rd) return k_sor_resident<Tc, kResNT, false, true, MODE>;
    return k_sor_resident<Tc, kResNT, false, false, MODE>;
}
template <class Tc>
ResidentFn<Tc> resident_kernel(const Brick& b) {
    if (b.mode == kResNarrow) return resident_kernel_m<Tc, kResNarrow>(b);
    if (b.mode == kResWide1) return resident_kernel_m<Tc, kResWide1>(b);
    return resident_kernel_m<Tc, kResWide>(b);
}

// Brick plan of the resident SOR kernel: the split of the (j,k) rows into at
// most (SM count) bricks that minimises the largest brick, under the shared
// memory limit (e of both colours for the brick and a one-row halo, plus d
// when it also fits).  Returns false when no plan fits one CTA per SM.
template <class Tc>
bool plan_resident(ntcfd_ctx* ctx) {
    const Geom& g = ctx->g;
    const int mx = ((g.nx + 3) >> 1) + 1;
    const size_t limit = ctx->smem_optin > 4096 ? ctx->smem_optin - 4096 : 0;
    long long best = -1;
    Brick bb{};
    size_t bsm = 0;
    for (int nbk = 1; nbk <= g.nz; ++nbk) {
        const int KB = (g.nz + nbk - 1) / nbk;
        const int nbk_eff = (g.nz + KB - 1) / KB;
        for (int nbj = 1; nbj <= g.ny; ++nbj) {
            const int JB = (g.ny + nbj - 1) / nbj;
            const int nbj_eff = (g.ny + JB - 1) / JB;
            if ((long long)nbj_eff * nbk_eff > ctx->sm_count) continue;
            Brick b{nbj_eff, nbk_eff, JB, KB, mx, 0, 0, res_mode(g.nx)};
            if (resident_smem<Tc>(b, g.nx) > limit) continue;
            // cache d, then rd, when they fit as well
            b.cache_d = 1;
            if (resident_smem<Tc>(b, g.nx) > limit) b.cache_d = 0;
            b.cache_rd = 1;
            if (resident_smem<Tc>(b, g.nx) > limit) b.cache_rd = 0;
            const long long cells = (long long)JB * KB;
            // smallest brick first, then the more cached arrays, then the smaller halo
            const long long score = cells * 1000000LL + (2 - b.cache_d - b.cache_rd) * 10000LL + (JB + KB);
            if (best < 0 || score < best) {
                best = score;
                bb = b;
                bsm = resident_smem<Tc>(b, g.nx);
            }
        }
    }
    if (best < 0) return false;
    auto kern = resident_kernel<Tc>(bb);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kResNT, bsm) != cudaSuccess ||
        per_sm < 1 || (long long)bb.nbj * bb.nbk > (long long)per_sm * ctx->sm_count) {
        cudaGetLastError();
        return false;
    }
    ctx->brick = bb;
    ctx->res_smem = bsm;
    ctx->res_grid = bb.nbj * bb.nbk;
    return true;
}

// K1 + K2 of the configured scheme on stream st, outside a graph: the
// Smagorinsky pass feeds only the QUICK_centre predictor; the other schemes
// evaluate their eddy viscosity inline.
void launch_predictor(ntcfd_ctx* ctx, cudaStream_t st) {
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    const bool qc = P.scheme == NTCFD_QUICK_CENTRE;
    if (P.LES && qc)
        k_smagorinsky<<<g3, b3, 0, st>>>(g, ctx->u, ctx->v, ctx->w, ctx->nut, P.Cs,
                                         P.smag_mode == NTCFD_SMAG_REF_ALIASED ? 1 : 0);
    const PredArgs pa{ctx->u, ctx->v, ctx->w, P.LES && qc ? ctx->nut : nullptr, ctx->us, ctx->vs, ctx->ws,
                      P.dt, 1. / P.Re, P.LES, ctx->fb, (long long)ctx->nat_elems};
    if (qc && P.precision == NTCFD_MIXED) {
        const int kc = p32_chunk(g.nx, g.ny, g.nz, ctx->p32_resident);
        k_predictor32<<<p32_grid(g, kc), dim3(kP32BX, kP32BY), p32_smem(kc), st>>>(g, ctx->tpf, pa, kc);
    } else if (qc) k_predictor<double><<<g3, b3, 0, st>>>(g, ctx->tpd, pa);
    else if (P.scheme == NTCFD_QUICK) k_predictor_scheme<kSchemeQuick><<<g3, b3, 0, st>>>(g, ctx->tpd, pa, P.Cs);
    else if (P.scheme == NTCFD_UPWIND) k_predictor_scheme<kSchemeUpwind><<<g3, b3, 0, st>>>(g, ctx->tpd, pa, P.Cs);
    else k_predictor_scheme<kSchemeCentre><<<g3, b3, 0, st>>>(g, ctx->tpd, pa, P.Cs);
}

// The step graph:
//   [K1 smag] -> K2 predictor -> K3a rhs -> begin -> WHILE(outer){ defect ->
//   WHILE(inner){ c x (red, black) -> check } -> correct -> outer_check } ->
//   K4 project -> K5 columns -> K5 total -> K6 x -> K6 y -> K6 z -> [divmax] -> end
// The step's nodes added to G (the step graph, or the body of the moving-body
// graph's IF node); `extra` kernels run before them in the same step.
template <class Tc>
int add_step_nodes(ntcfd_ctx* ctx, cudaGraph_t G, int extra) {
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    std::vector<cudaGraphNode_t> dep;
    cudaGraphNode_t n;
    const bool qc = P.scheme == NTCFD_QUICK_CENTRE;
    if (P.LES && qc) {
        GK(add_kernel(&n, G, dep, k_smagorinsky, g3, b3, g, (const double*)ctx->u,
                      (const double*)ctx->v, (const double*)ctx->w, ctx->nut, P.Cs,
                      P.smag_mode == NTCFD_SMAG_REF_ALIASED ? 1 : 0));
        dep = {n};
    }
    PredArgs pa{ctx->u, ctx->v, ctx->w, P.LES && qc ? ctx->nut : nullptr, ctx->us, ctx->vs, ctx->ws,
                P.dt, 1. / P.Re, P.LES, ctx->fb, (long long)ctx->nat_elems};
    if (qc && P.precision == NTCFD_MIXED) {
        const int kc = p32_chunk(g.nx, g.ny, g.nz, ctx->p32_resident);
        GK(add_kernel_ex(&n, G, dep, k_predictor32, p32_grid(g, kc), dim3(kP32BX, kP32BY), p32_smem(kc), false,
                         g, ctx->tpf, pa, kc));
    } else if (qc) GK(add_kernel(&n, G, dep, k_predictor<double>, g3, b3, g, ctx->tpd, pa));
    else if (P.scheme == NTCFD_QUICK)
        GK(add_kernel(&n, G, dep, k_predictor_scheme<kSchemeQuick>, g3, b3, g, ctx->tpd, pa, P.Cs));
    else if (P.scheme == NTCFD_UPWIND)
        GK(add_kernel(&n, G, dep, k_predictor_scheme<kSchemeUpwind>, g3, b3, g, ctx->tpd, pa, P.Cs));
    else
        GK(add_kernel(&n, G, dep, k_predictor_scheme<kSchemeCentre>, g3, b3, g, ctx->tpd, pa, P.Cs));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_rhs, walk_grid(g, ctx->sm_count), walk_block(), g, ctx->scd, (const double*)ctx->u,
                  (const double*)ctx->v, (const double*)ctx->w, (const double*)ctx->us,
                  (const double*)ctx->vs, (const double*)ctx->ws, ctx->b, P.dt, back_iface(ctx)));
    dep = {n};
    ctx->resident = false;
    if (P.sor_path != NTCFD_SOR_STREAMING) {
        ctx->resident = plan_resident<Tc>(ctx);
        if (!ctx->resident && P.sor_path == NTCFD_SOR_RESIDENT)
            return fail(ctx, NTCFD_EINVAL, "the resident SOR kernel does not fit this grid on this device");
    }
    if (ctx->resident) {
        // the resident kernel runs the whole solve (every correction cycle), so the
        // solve is two plain nodes: the defect (which also starts the solve) and the kernel
        Tc *eR = (Tc*)ctx->eR, *eB = (Tc*)ctx->eB, *dR = (Tc*)ctx->dR, *dB = (Tc*)ctx->dB;
        GK(add_kernel(&n, G, dep, k_defect<Tc>, g3, b3, g, ctx->scd, (const double*)ctx->p,
                      (const double*)ctx->b, dR, dB, eR, eB, (const Tc*)ctx->rdR, (const Tc*)ctx->rdB, ctx->ctl,
                      (cudaGraphConditionalHandle)0, 0, ctx->ring, (unsigned int*)ctx->bar, 1, 0));
        dep = {n};
        GK(add_kernel_ex(&n, G, dep, resident_kernel<Tc>(ctx->brick), dim3(ctx->res_grid), dim3(kResNT),
                         ctx->res_smem, true, g, sor_coef<Tc>(ctx), ctx->brick, ctx->p, (const double*)ctx->b,
                         eR, eB, dR, dB, (const Tc*)ctx->rdR, (const Tc*)ctx->rdB, ctx->ctl,
                         ctx->bar, P.omega, P.zeta, P.itmax, ctx->cycle_len, ctx->csweeps, ctx->ring));
        dep = {n};
    } else {
        cudaGraphConditionalHandle hout, hin;
        GK(cudaGraphConditionalHandleCreate(&hout, G, 0, 0));
        GK(add_kernel(&n, G, dep, k_sor_begin, dim3(1), dim3(1), ctx->ctl, P.itmax, hout, 1));
        dep = {n};
        cudaGraph_t outer;
        GK(add_while(&n, G, dep, hout, &outer));
        dep = {n};
        GK(cudaGraphConditionalHandleCreate(&hin, outer, 0, 0));
        std::vector<cudaGraphNode_t> od;
        cudaGraphNode_t m;
        Tc *eR = (Tc*)ctx->eR, *eB = (Tc*)ctx->eB, *dR = (Tc*)ctx->dR, *dB = (Tc*)ctx->dB;
        // the defect of p (first cycle) or its update from the last cycle's e (later
        // cycles, as the resident kernel restarts); the row sweep (FP32) reads e as 0 in
        // a cycle's first sweep, the column sweep (FP64) after k_clear_e
        GK(add_kernel(&m, outer, od, k_defect_rows<Tc, kSweepNT>, sweep_grid(g, kSweepNT, ctx->defect_resident),
                      dim3(kSweepNT), g, ctx->scd, sor_coef<Tc>(ctx), ctx->p,
                      (const double*)ctx->b, dR, dB, (const Tc*)eR, (const Tc*)eB, ctx->ctl, hin, 1));
        od = {m};
        if (!kRowSweep<Tc>) {
            GK(add_kernel(&m, outer, od, k_clear_e<Tc>, g3, b3, g, eR, eB));
            od = {m};
        }
        cudaGraph_t inner;
        GK(add_while(&m, outer, od, hin, &inner));
        od = {m};
        {
            std::vector<cudaGraphNode_t> id;
            cudaGraphNode_t s;
            const SorCoef<Tc> sc = sor_coef<Tc>(ctx);
            const dim3 bs = Sweep<Tc>::block(), gs = Sweep<Tc>::grid(g, ctx->row_resident);
            const Ctl* cctl = ctx->ctl;
            for (int sub = 0; sub < ctx->csweeps; ++sub) {
                GK(add_kernel(&s, inner, id, Sweep<Tc>::fn, gs, bs, g, sc,
                              eR, (const Tc*)eB, (const Tc*)dR, (const Tc*)ctx->rdR, 0, P.omega, cctl,
                              sub, P.itmax,
                              ctx->cycle_len, ctx->csweeps > 1 ? 1 : 0, ctx->slots, kRowSweep<Tc> ? 1 : 0));
                id = {s};
                GK(add_kernel(&s, inner, id, Sweep<Tc>::fn, gs, bs, g, sc,
                              eB, (const Tc*)eR, (const Tc*)dB, (const Tc*)ctx->rdB, 1, P.omega, cctl,
                              sub, P.itmax,
                              ctx->cycle_len, ctx->csweeps > 1 ? 1 : 0, ctx->slots, kRowSweep<Tc> ? 1 : 0));
                id = {s};
            }
            GK(add_kernel(&s, inner, id, k_sor_check, dim3(1), dim3(32), ctx->ctl, ctx->slots,
                          ctx->csweeps, P.itmax, ctx->cycle_len, P.zeta, hin, 1));
        }
        GK(add_kernel(&m, outer, od, k_outer_check, dim3(1), dim3(1), ctx->ctl, P.itmax, hout, 1));
        // the last cycle's e (k_defect_rows adds the earlier ones)
        GK(add_kernel(&n, G, dep, k_correct_last<Tc>, g3, b3, g, ctx->p, (const Tc*)eR, (const Tc*)eB,
                      (const Ctl*)ctx->ctl));
        dep = {n};
    }
    ProjArgs pj{ctx->u, ctx->v, ctx->w, ctx->us, ctx->vs, ctx->ws, ctx->p, ctx->eta, ctx->partZ,
                ctx->partY, P.dt, P.u_solid[0], P.u_solid[1], P.u_solid[2], kProjKc};
    GK(add_kernel(&n, G, dep, k_project, dim3((g.nx + 31) / 32, (g.ny + 3) / 4, ctx->nchunk),
                  dim3(32, 4, 1), g, pj));
    dep = {n};
    // the force integral only where a mask can make forces (ETA = 0: zero by construction)
    if (ctx->mask_nonzero) {
        GK(add_kernel(&n, G, dep, k_force_columns, dim3(296), dim3(256), g, (const double*)ctx->partZ,
                      (const double*)ctx->partY, ctx->nchunk, ctx->FXz, ctx->FYz));
        dep = {n};
        GK(add_kernel(&n, G, dep, k_force_total<256>, dim3((g.nx + 7) / 8), dim3(256), g, (const double*)ctx->FXz,
                      (const double*)ctx->FYz, ctx->FXy, ctx->FYy, P.lx, ctx->ctl, ctx->fdone, ctx->rec));
        dep = {n};
    }
    BcArgs ba{};
    ba.u = ctx->u; ba.v = ctx->v; ba.w = ctx->w; ba.p = ctx->p;
    std::memcpy(ba.bc, P.bc, sizeof ba.bc);
    std::memcpy(ba.val, P.bc_value, sizeof ba.val);
    ba.faceW = ctx->faceW; ba.faceE = ctx->faceE; ba.faceS = ctx->faceS;
    ba.faceN = ctx->faceN; ba.faceB = ctx->faceB; ba.faceF = ctx->faceF;
    GK(add_kernel(&n, G, dep, k_bc_x, bc_grid_x(g), dim3(32, 8), g, ba));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_bc_y, bc_grid_y(g), dim3(32, 8), g, ba));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_bc_z, bc_grid_z(g), dim3(32, 8), g, ba));
    dep = {n};
    if (P.diag_divergence) {
        GK(add_kernel(&n, G, dep, k_divmax<256>, g3, b3, g, (const double*)ctx->u,
                      (const double*)ctx->v, (const double*)ctx->w, ctx->divslot));
        dep = {n};
    }
    // kernels of a step: predictor, rhs, project, force (2, with a mask), bc (3), step_end, + LES,
    // + diagnostic; + sor_begin, the final correction and 2 per cycle (streaming FP32; 3 with
    // the FP64 clear) or 2 per solve (resident)
    const int fixed = extra + 7 + (ctx->mask_nonzero ? 2 : 0) + (P.LES ? 1 : 0) + (P.diag_divergence ? 1 : 0) +
                      (ctx->resident ? 0 : 2);
    GK(add_kernel(&n, G, dep, k_step_end, dim3(1), dim3(1), ctx->ctl, ctx->rec, ctx->divslot,
                  P.diag_divergence, fixed, ctx->resident ? 2 : (kRowSweep<Tc> ? 2 : 3),
                  ctx->resident ? 0 : 2 * ctx->csweeps + 1, ctx->mask_nonzero ? 1 : 0, P.lx));
    return 0;
}

template <class Tc>
int build_graph(ntcfd_ctx* ctx) {
    cudaGraph_t G;
    GK(cudaGraphCreate(&G, 0));
    ctx->graph = G;
    if (int rc = add_step_nodes<Tc>(ctx, G, 0)) return rc;
    GK(cudaGraphInstantiate(&ctx->exec, G, 0));
    return 0;
}

// Kernels of the moving body's mask in a step of the moving-body graph.
constexpr int kDynKernels = 7;

// The moving-body step graph (ntcfd_set_dynamic_aoa): the step's mask
// (airfoil.f90:311-321, RayCasting at the step's angle) -> gate -> IF(no tie in
// this call){ the step }.
template <class Tc>
int build_dyn_graph(ntcfd_ctx* ctx) {
    const Geom g = ctx->g;
    cudaGraph_t G;
    GK(cudaGraphCreate(&G, 0));
    ctx->graph_dyn = G;
    const DynMask m = ctx->dyn;
    const Ctl* cctl = ctx->ctl;
    const int cells = g.ny * g.nz;
    std::vector<cudaGraphNode_t> dep;
    cudaGraphNode_t n;
    GK(add_kernel(&n, G, dep, k_dyn_rotate<512>, dim3(1), dim3(512), g.ny, g.nz, (const double*)ctx->coordY,
                  (const double*)ctx->coordZ, m, cctl));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_dyn_main, dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), g.ny, g.nz,
                  (const double*)ctx->coordY, (const double*)ctx->coordZ, m, cctl));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_dyn_points, dim3((m.npts + 127) / 128), dim3(128), g.ny, g.nz,
                  (const double*)ctx->coordY, (const double*)ctx->coordZ, m, cctl));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_dyn_compact, dim3((cells + 255) / 256), dim3(256), cells, m, cctl));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_dyn_sub<256>, dim3(2 * ctx->sm_count), dim3(256), g.nz,
                  (const double*)ctx->coordY, (const double*)ctx->coordZ, m, cctl));
    dep = {n};
    GK(add_kernel(&n, G, dep, k_dyn_extrude, dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2),
                  dim3(32, 4, 2), g, (const double*)m.eta1, ctx->eta, cctl));
    dep = {n};
    cudaGraphConditionalHandle h;
    GK(cudaGraphConditionalHandleCreate(&h, G, 0, 0));
    GK(add_kernel(&n, G, dep, k_dyn_gate, dim3(1), dim3(1), m, ctx->ctl, h));
    dep = {n};
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    GK(cudaGraphAddNode(&n, G, dep.data(), dep.size(), &np));
    if (int rc = add_step_nodes<Tc>(ctx, np.conditional.phGraph_out[0], kDynKernels)) return rc;
    GK(cudaGraphInstantiate(&ctx->exec_dyn, G, 0));
    return 0;
}

// One SOR solve launched from the host: the graph's loop structure (defect-
// correction cycles around the resident kernel or around streaming sweeps
// with a stop test every check_every sweeps), on pressure `p` (interior
// updated, ghosts read) with right-hand side `b`, stop rule max|change| <=
// zeta, sweep cap itmax and relaxation omega.  *hc receives the final
// control block.  With chunk > 1 the streaming path queues up to `chunk` loop
// bodies (and at most a cycle's) before the host reads the control block:
// the bodies queued after the stop do nothing (their sweeps skip, their
// tests return), so the solve is the same with one host round trip per chunk
// instead of one per body.  chunk = 1 keeps the graph's launches one for one.
template <class Tc>
int sor_solve_eager(ntcfd_ctx* ctx, double* p, const double* b, double zeta, int itmax, double omega, Ctl* hc,
                    int chunk = 1) {
    const Geom g = ctx->g;
    cudaStream_t st = ctx->stream;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    Tc *eR = (Tc*)ctx->eR, *eB = (Tc*)ctx->eB, *dR = (Tc*)ctx->dR, *dB = (Tc*)ctx->dB;
    const SorCoef<Tc> sc = sor_coef<Tc>(ctx);
    Ctl& h = *hc;
    h = Ctl{};
    auto read_ctl = [&]() -> int {
        CK(cudaMemcpyAsync(&h, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        return 0;
    };
    if (ctx->resident) {
        // one defect (starting the solve) and one launch that runs every cycle
        k_defect<Tc><<<g3, b3, 0, st>>>(g, ctx->scd, p, b, dR, dB, eR, eB, (const Tc*)ctx->rdR,
                                        (const Tc*)ctx->rdB, ctx->ctl, 0, 0, ctx->ring, (unsigned int*)ctx->bar, 1, 0);
        void* args[] = {(void*)&g, (void*)&sc, (void*)&ctx->brick, (void*)&p, (void*)&b, (void*)&eR,
                        (void*)&eB, (void*)&dR, (void*)&dB, (void*)&ctx->rdR, (void*)&ctx->rdB,
                        (void*)&ctx->ctl, (void*)&ctx->bar, (void*)&omega, (void*)&zeta,
                        (void*)&itmax, (void*)&ctx->cycle_len, (void*)&ctx->csweeps, (void*)&ctx->ring};
        CK(cudaLaunchCooperativeKernel((const void*)resident_kernel<Tc>(ctx->brick), dim3(ctx->res_grid),
                                       dim3(kResNT), args, ctx->res_smem, st));
        if (int rc = read_ctl()) return rc;
        CK(cudaGetLastError());
        return 0;
    }
    k_sor_begin<<<1, 1, 0, st>>>(ctx->ctl, itmax, 0, 0);
    bool more = itmax > 0;
    const int big_guard = ctx->csweeps > 1 || chunk > 1 ? 1 : 0;
    const int cycle_bodies = std::max(1, ctx->cycle_len / ctx->csweeps);
    const int queued = std::max(1, std::min(chunk, cycle_bodies));
    while (more) {
        {
            k_defect_rows<Tc, kSweepNT><<<sweep_grid(g, kSweepNT, ctx->defect_resident), kSweepNT, 0, st>>>(
                g, ctx->scd, sc, p, b, dR, dB, eR, eB, ctx->ctl, 0, 0);
            if (!kRowSweep<Tc>) k_clear_e<Tc><<<g3, b3, 0, st>>>(g, eR, eB);
            const dim3 bs = Sweep<Tc>::block(), gs = Sweep<Tc>::grid(g, ctx->row_resident);
            for (;;) {
                for (int q = 0; q < queued; ++q) {
                    for (int sub = 0; sub < ctx->csweeps; ++sub) {
                        Sweep<Tc>::fn<<<gs, bs, 0, st>>>(
                            g, sc, eR, eB, dR, (const Tc*)ctx->rdR, 0, omega, ctx->ctl, sub, itmax,
                            ctx->cycle_len, big_guard, ctx->slots, kRowSweep<Tc> ? 1 : 0);
                        Sweep<Tc>::fn<<<gs, bs, 0, st>>>(
                            g, sc, eB, eR, dB, (const Tc*)ctx->rdB, 1, omega, ctx->ctl, sub, itmax,
                            ctx->cycle_len, big_guard, ctx->slots, kRowSweep<Tc> ? 1 : 0);
                    }
                    k_sor_check<<<1, 32, 0, st>>>(ctx->ctl, ctx->slots, ctx->csweeps, itmax, ctx->cycle_len,
                                                  zeta, 0, 0);
                }
                if (int rc = read_ctl()) return rc;
                if (h.pad_stop) break;
            }
        }
        k_outer_check<<<1, 1, 0, st>>>(ctx->ctl, itmax, 0, 0);
        if (int rc = read_ctl()) return rc;
        more = h.pad_more != 0;
    }
    // the last cycle's e (k_defect_rows adds the earlier ones)
    k_correct_last<Tc><<<g3, b3, 0, st>>>(g, p, eR, eB, ctx->ctl);
    CK(cudaGetLastError());
    return 0;
}

// One step with every kernel launched from the host (no CUDA graph): the
// same kernels and loop decisions as the graph, for kernel profilers (which
// cannot look inside graphs that contain conditional nodes) and debugging.
template <class Tc>
int run_step_eager(ntcfd_ctx* ctx) {
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    cudaStream_t st = ctx->stream;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    launch_predictor(ctx, st);
    k_rhs<<<walk_grid(g, ctx->sm_count), walk_block(), 0, st>>>(g, ctx->scd, ctx->u, ctx->v, ctx->w, ctx->us, ctx->vs, ctx->ws, ctx->b, P.dt, back_iface(ctx));
    Ctl h{};
    if (int rc = sor_solve_eager<Tc>(ctx, ctx->p, ctx->b, P.zeta, P.itmax, P.omega, &h)) return rc;
    ProjArgs pj{ctx->u, ctx->v, ctx->w, ctx->us, ctx->vs, ctx->ws, ctx->p, ctx->eta, ctx->partZ,
                ctx->partY, P.dt, P.u_solid[0], P.u_solid[1], P.u_solid[2], kProjKc};
    k_project<<<dim3((g.nx + 31) / 32, (g.ny + 3) / 4, ctx->nchunk), dim3(32, 4, 1), 0, st>>>(g, pj);
    if (ctx->mask_nonzero) {
        k_force_columns<<<296, 256, 0, st>>>(g, ctx->partZ, ctx->partY, ctx->nchunk, ctx->FXz, ctx->FYz);
        k_force_total<256><<<(g.nx + 7) / 8, 256, 0, st>>>(g, ctx->FXz, ctx->FYz, ctx->FXy, ctx->FYy, P.lx,
                                                              ctx->ctl, ctx->fdone, ctx->rec);
    }
    BcArgs ba{};
    ba.u = ctx->u; ba.v = ctx->v; ba.w = ctx->w; ba.p = ctx->p;
    std::memcpy(ba.bc, P.bc, sizeof ba.bc);
    std::memcpy(ba.val, P.bc_value, sizeof ba.val);
    ba.faceW = ctx->faceW; ba.faceE = ctx->faceE; ba.faceS = ctx->faceS;
    ba.faceN = ctx->faceN; ba.faceB = ctx->faceB; ba.faceF = ctx->faceF;
    k_bc_x<<<bc_grid_x(g), dim3(32, 8), 0, st>>>(g, ba);
    k_bc_y<<<bc_grid_y(g), dim3(32, 8), 0, st>>>(g, ba);
    k_bc_z<<<bc_grid_z(g), dim3(32, 8), 0, st>>>(g, ba);
    if (P.diag_divergence) k_divmax<256><<<g3, b3, 0, st>>>(g, ctx->u, ctx->v, ctx->w, ctx->divslot);
    const int fixed = 7 + (ctx->mask_nonzero ? 2 : 0) + (P.LES ? 1 : 0) + (P.diag_divergence ? 1 : 0) +
                      (ctx->resident ? 0 : 2);
    k_step_end<<<1, 1, 0, st>>>(ctx->ctl, ctx->rec, ctx->divslot, P.diag_divergence, fixed,
                                ctx->resident ? 2 : (kRowSweep<Tc> ? 2 : 3), ctx->resident ? 0 : 2 * ctx->csweeps + 1,
                                ctx->mask_nonzero ? 1 : 0, P.lx);
    CK(cudaGetLastError());
    return 0;
}

int validate(const ntcfd_params* p, std::string* why) {
    char b[256];
    auto bad = [&](const char* m) { *why = m; return NTCFD_EINVAL; };
    if (p->nx < 3 || p->ny < 3 || p->nz < 3) return bad("nx, ny, nz must be >= 3");
    if (!(p->Re > 0) || !(p->dt > 0)) return bad("Re and dt must be positive");
    if (!(p->omega > 0 && p->omega < 2)) return bad("omega must lie in (0, 2)");
    if (p->itmax < 0) return bad("itmax must be >= 0");
    if (!(p->zeta >= 0)) return bad("zeta must be >= 0");
    if (p->precision != NTCFD_FP64 && p->precision != NTCFD_MIXED) return bad("precision must be NTCFD_FP64 or NTCFD_MIXED");
    if (p->sor_order != NTCFD_SOR_REDBLACK)
        return bad("the device solver is red-black SOR (sor_order = NTCFD_SOR_REDBLACK)");
    if (p->scheme < NTCFD_QUICK_CENTRE || p->scheme > NTCFD_CENTRE)
        return bad("scheme must be NTCFD_QUICK_CENTRE, NTCFD_QUICK, NTCFD_UPWIND or NTCFD_CENTRE");
    if (p->sor_path < NTCFD_SOR_AUTO || p->sor_path > NTCFD_SOR_RESIDENT) return bad("bad sor_path");
    if (p->eager != 0 && p->eager != 1) return bad("eager must be 0 or 1");
    if (p->smag_mode != NTCFD_SMAG_REF_ALIASED && p->smag_mode != NTCFD_SMAG_STAGGERED) return bad("bad smag_mode");
    if (p->LES != 0 && p->LES != 1) return bad("LES must be 0 or 1");
    if (p->check_every < 0 || p->mixed_cycle < 0) return bad("check_every and mixed_cycle must be >= 0");
    for (int wl = 0; wl < 6; ++wl)
        for (int c = 0; c < 3; ++c) {
            if (p->bc[wl][c] < 0 || p->bc[wl][c] > NTCFD_BC_INTERFACE) return bad("bad boundary-condition kind");
            if (p->bc[wl][c] == NTCFD_BC_INTERFACE && (wl < NTCFD_BACK || p->bc[wl][0] != p->bc[wl][1] ||
                                                       p->bc[wl][0] != p->bc[wl][2]))
                return bad("NTCFD_BC_INTERFACE: Back or Front walls only, all three components");
        }
    for (int ax = 0; ax < 3; ++ax) {
        const int lo = 2 * ax, hi = 2 * ax + 1;
        bool any = false, all = true;
        for (int c = 0; c < 3; ++c) {
            for (int wl : {lo, hi}) {
                const bool per = p->bc[wl][c] == NTCFD_BC_PERIODIC;
                any = any || per;
                all = all && per;
            }
        }
        if (any && !all) {
            snprintf(b, sizeof b, "periodic axis %d: both walls and all three components must be periodic", ax);
            *why = b;
            return NTCFD_EINVAL;
        }
    }
    for (size_t q = 0; q < sizeof p->reserved / sizeof p->reserved[0]; ++q)
        if (p->reserved[q] != 0) return bad("reserved fields must be zero");
    return 0;
}

template <class T>
void make_axis_tables(int n, const double* iD, const double* Ds, T* out /* 6 x (n+5) */,
                      AxisTabs<T>* at, T** base_for_ptrs) {
    // out layout: riD, rDs, As, Bs, Ac, Bc, each n+5 entries, entry q <-> index q-2
    const int L = n + 5;
    auto I = [&](const double* a, int i) { return a[i + 1]; };   // a(-1:n+2) from index 0
    for (int q = 0; q < 6 * L; ++q) out[q] = T(0);
    for (int i = -1; i <= n + 2; ++i) {
        out[0 * L + i + 2] = (T)(1.0 / I(iD, i));
        out[1 * L + i + 2] = (T)(1.0 / I(Ds, i));
    }
    for (int a = -1; a <= n + 1; ++a) {
        const double h1 = I(iD, a + 1);
        out[2 * L + a + 2] = (T)(0.125 * h1 * h1 / I(Ds, a));
        out[3 * L + a + 2] = (T)(0.125 * h1 * h1 / I(Ds, a + 1));
        const double H = I(Ds, a);
        out[4 * L + a + 2] = (T)(0.125 * H * H / I(iD, a));
        out[5 * L + a + 2] = (T)(0.125 * H * H / I(iD, a + 1));
    }
    (void)at;
    (void)base_for_ptrs;
}

}  // namespace

namespace {

template <class Tc>
int time_kernels_t(ntcfd_ctx* ctx, int reps, ntcfd_kernel_times* out) {
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    float ms = 0.0f;
    auto timed = [&](auto&& launch, float* dst, int per) -> int {
        launch();  // warm-up
        CK(cudaEventRecord(ctx->ev0, ctx->stream));
        for (int r = 0; r < reps; ++r) launch();
        CK(cudaEventRecord(ctx->ev1, ctx->stream));
        CK(cudaEventSynchronize(ctx->ev1));
        CK(cudaGetLastError());
        CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
        *dst = ms / (float)(reps * per);
        return 0;
    };
    int rc;
    if ((rc = timed([&] { launch_predictor(ctx, ctx->stream); }, &out->predictor_ms, 1)))
        return rc;
    if ((rc = timed([&] {
             k_rhs<<<walk_grid(g, ctx->sm_count), walk_block(), 0, ctx->stream>>>(g, ctx->scd, ctx->u, ctx->v, ctx->w, ctx->us, ctx->vs,
                                               ctx->ws, ctx->b, P.dt, back_iface(ctx));
         }, &out->rhs_ms, 1)))
        return rc;
    Tc *eR = (Tc*)ctx->eR, *eB = (Tc*)ctx->eB, *dR = (Tc*)ctx->dR, *dB = (Tc*)ctx->dB;
    // the defect the path's restarts use: k_defect (resident), k_defect_rows (streaming)
    if ((rc = timed([&] {
             if (ctx->resident)
                 k_defect<Tc><<<g3, b3, 0, ctx->stream>>>(g, ctx->scd, ctx->p, ctx->b, dR, dB, eR, eB,
                                                          (const Tc*)ctx->rdR, (const Tc*)ctx->rdB, ctx->ctl, 0, 0,
                                                          nullptr, nullptr, 0, 0);
             else
                 // on scratch (us is rewritten by the predictor every step): from a
                 // cycle on, the restart also adds e to the p it is given
                 k_defect_rows<Tc, kSweepNT><<<sweep_grid(g, kSweepNT, ctx->defect_resident), kSweepNT, 0,
                                               ctx->stream>>>(g, ctx->scd, sor_coef<Tc>(ctx), ctx->us, ctx->b, dR,
                                                              dB, eR, eB, ctx->ctl, 0, 0);
         }, &out->defect_ms, 1)))
        return rc;
    const SorCoef<Tc> sc = sor_coef<Tc>(ctx);
    const dim3 bs = Sweep<Tc>::block(), gs = Sweep<Tc>::grid(g, ctx->row_resident);
    const int big = 1 << 30;
    if ((rc = timed([&] {
             Sweep<Tc>::fn<<<gs, bs, 0, ctx->stream>>>(
                 g, sc, eR, eB, dR, (const Tc*)ctx->rdR, 0, P.omega, ctx->ctl, 0, big, big, 0, ctx->slots, 0);
             Sweep<Tc>::fn<<<gs, bs, 0, ctx->stream>>>(
                 g, sc, eB, eR, dB, (const Tc*)ctx->rdB, 1, P.omega, ctx->ctl, 0, big, big, 0, ctx->slots, 0);
         }, &out->sweep_ms, 2)))
        return rc;
    // the resident kernel: one launch of `nsw` sweeps (zeta = 0, one cycle) on a scratch
    // copy of p, less a launch of no sweep (the defect before it, the kernel's set-up and
    // p += e)
    if (ctx->resident) {
        const int nsw = 50;
        double* pscratch = ctx->us;   // rewritten by the predictor every step
        CK(cudaMemcpyAsync(pscratch, ctx->p, ctx->nat_elems * sizeof(double), cudaMemcpyDeviceToDevice,
                           ctx->stream));
        auto resident = [&](const int* sweeps) {
            k_defect<Tc><<<g3, b3, 0, ctx->stream>>>(g, ctx->scd, pscratch, ctx->b, dR, dB, eR, eB,
                                                     (const Tc*)ctx->rdR, (const Tc*)ctx->rdB, ctx->ctl, 0, 0,
                                                     ctx->ring, (unsigned int*)ctx->bar, 1, 0);
            void* args[] = {(void*)&g, (void*)&sc, (void*)&ctx->brick, (void*)&pscratch, (void*)&ctx->b,
                            (void*)&eR, (void*)&eB, (void*)&dR, (void*)&dB, (void*)&ctx->rdR, (void*)&ctx->rdB,
                            (void*)&ctx->ctl, (void*)&ctx->bar, (void*)&P.omega, (void*)&kZeroZeta,
                            (void*)sweeps, (void*)sweeps, (void*)&kOne, (void*)&ctx->ring};
            cudaLaunchCooperativeKernel((const void*)resident_kernel<Tc>(ctx->brick), dim3(ctx->res_grid),
                                        dim3(kResNT), args, ctx->res_smem, ctx->stream);
        };
        const int none = 0;
        float t0 = 0.0f;
        if ((rc = timed([&] { resident(&none); }, &t0, 1))) return rc;
        if ((rc = timed([&] { resident(&nsw); }, &out->resident_ms, 1))) return rc;
        out->resident_ms -= t0;
        out->resident_sweeps = (float)nsw;
    }
    // K4 on the predicted velocity in place (us/vs/ws are rewritten every step)
    ProjArgs pj{ctx->us, ctx->vs, ctx->ws, ctx->us, ctx->vs, ctx->ws, ctx->p, ctx->eta, ctx->partZ,
                ctx->partY, P.dt, P.u_solid[0], P.u_solid[1], P.u_solid[2], kProjKc};
    if ((rc = timed([&] {
             k_project<<<dim3((g.nx + 31) / 32, (g.ny + 3) / 4, ctx->nchunk), dim3(32, 4, 1), 0,
                         ctx->stream>>>(g, pj);
         }, &out->project_ms, 1)))
        return rc;
    // K6 is idempotent on the state; the saved faces go to scratch here
    BcArgs ba{};
    ba.u = ctx->u; ba.v = ctx->v; ba.w = ctx->w; ba.p = ctx->p;
    std::memcpy(ba.bc, P.bc, sizeof ba.bc);
    std::memcpy(ba.val, P.bc_value, sizeof ba.val);
    double* junk = ctx->outbuf;
    const size_t nxy = (size_t)g.nx * g.ny, nxz = (size_t)g.nx * g.nz;
    ba.faceW = junk; ba.faceE = junk + (size_t)g.ny * g.nz; ba.faceS = ba.faceE + (size_t)g.ny * g.nz;
    ba.faceN = ba.faceS + nxz; ba.faceB = ba.faceN + nxz; ba.faceF = ba.faceB + nxy;
    if ((rc = timed([&] {
             k_bc_x<<<bc_grid_x(g), dim3(32, 8), 0, ctx->stream>>>(g, ba);
             k_bc_y<<<bc_grid_y(g), dim3(32, 8), 0, ctx->stream>>>(g, ba);
             k_bc_z<<<bc_grid_z(g), dim3(32, 8), 0, ctx->stream>>>(g, ba);
         }, &out->bc_ms, 1)))
        return rc;
    return 0;
}

}  // namespace

// =====================================================================  ABI
extern "C" {

void ntcfd_default_params(ntcfd_params* p) {
    std::memset(p, 0, sizeof *p);
    p->nx = p->ny = p->nz = 40;
    p->Re = 10.0;
    p->dt = (double)1.0e-3f;      // real*8 parameter initialised from a default-real literal
    p->omega = 1.5;
    p->zeta = (double)1.e-4f;
    p->itmax = 3000;
    p->LES = 0;
    p->Cs = (double)0.18f;
    p->scheme = NTCFD_QUICK_CENTRE;
    p->precision = NTCFD_FP64;
    p->sor_order = NTCFD_SOR_REDBLACK;
    p->smag_mode = NTCFD_SMAG_REF_ALIASED;
    p->check_every = 1;
    for (int wl = 0; wl < 6; ++wl)
        for (int c = 0; c < 3; ++c) {
            p->bc[wl][c] = NTCFD_BC_NOSLIP;
            p->bc_value[wl][c] = 1.0;
        }
    p->bc[NTCFD_NORTH][2] = NTCFD_BC_DIRICHLET;   // NorthWall_w = 'Dirichlet'
    p->lx = 1.0;
}

int ntcfd_create(const ntcfd_params* prm, ntcfd_ctx** out) {
    if (!prm || !out) return NTCFD_EINVAL;
    *out = nullptr;
    std::string why;
    ntcfd_ctx* ctx = new ntcfd_ctx();
    if (int rc = validate(prm, &why)) {
        // a context is still returned so that ntcfd_last_error can explain the failure
        ctx->err = why;
        *out = ctx;
        return rc;
    }
    ctx->prm = *prm;
    ntcfd_params& P = ctx->prm;
    if (P.check_every == 0) P.check_every = 1;
    ctx->csweeps = P.check_every;
    // sweeps per defect-correction cycle: mixed_cycle when set, else kMixedCycle for
    // MIXED (FP32 sweeps) and one cycle for FP64
    const bool cycles = P.mixed_cycle > 0 || P.precision == NTCFD_MIXED;
    int cl = P.mixed_cycle > 0 ? P.mixed_cycle : (P.precision == NTCFD_MIXED ? kMixedCycle : P.itmax);
    if (cycles && cl % ctx->csweeps) cl += ctx->csweeps - cl % ctx->csweeps;
    ctx->cycle_len = cl > 0 ? cl : 1;
    *out = ctx;
    CK(cudaSetDevice(P.device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ctx->ev0));
    CK(cudaEventCreate(&ctx->ev1));
    Geom& g = ctx->g;
    g.nx = P.nx; g.ny = P.ny; g.nz = P.nz;
    g.px = ((P.nx + 10) + 7) & ~7;
    g.py = P.ny + 4;
    g.pz = (long long)g.px * g.py;
    g.mxp = ((((P.nx + 3) >> 1) + 1) + 7) & ~7;
    g.mz = (long long)g.mxp * g.py;
    ctx->nat_elems = (size_t)g.pz * (P.nz + 4);
    ctx->spl_elems = (size_t)g.mz * (P.nz + 4);
    const size_t N = ctx->nat_elems;
    int rc;
    double** nat[] = {&ctx->u, &ctx->v, &ctx->w, &ctx->p, &ctx->us, &ctx->vs, &ctx->ws, &ctx->b, &ctx->eta};
    for (double** a : nat)
        if ((rc = dalloc(ctx, a, N))) return rc;
    if (P.LES && (rc = dalloc(ctx, &ctx->nut, N))) return rc;
    const size_t esz = P.precision == NTCFD_MIXED ? sizeof(float) : sizeof(double);
    void** spl[] = {&ctx->eR, &ctx->eB, &ctx->dR, &ctx->dB, &ctx->rdR, &ctx->rdB};
    for (void** a : spl) {
        char* q;
        if ((rc = dalloc(ctx, &q, ctx->spl_elems * esz))) return rc;
        *a = q;
    }
    ctx->nchunk = (P.nz + kProjKc - 1) / kProjKc;
    const size_t cols = (size_t)P.nx * P.ny;
    if ((rc = dalloc(ctx, &ctx->partZ, cols * ctx->nchunk))) return rc;
    if ((rc = dalloc(ctx, &ctx->partY, cols * ctx->nchunk))) return rc;
    if ((rc = dalloc(ctx, &ctx->FXz, cols))) return rc;
    if ((rc = dalloc(ctx, &ctx->FYz, cols))) return rc;
    if ((rc = dalloc(ctx, &ctx->FXy, (size_t)P.nx))) return rc;
    if ((rc = dalloc(ctx, &ctx->FYy, (size_t)P.nx))) return rc;
    if ((rc = dalloc(ctx, &ctx->fdone, 1))) return rc;
    if ((rc = dalloc(ctx, &ctx->faceW, (size_t)P.ny * P.nz))) return rc;
    if ((rc = dalloc(ctx, &ctx->faceE, (size_t)P.ny * P.nz))) return rc;
    if ((rc = dalloc(ctx, &ctx->faceS, (size_t)P.nx * P.nz))) return rc;
    if ((rc = dalloc(ctx, &ctx->faceN, (size_t)P.nx * P.nz))) return rc;
    if ((rc = dalloc(ctx, &ctx->faceB, (size_t)P.nx * P.ny))) return rc;
    if ((rc = dalloc(ctx, &ctx->faceF, (size_t)P.nx * P.ny))) return rc;
    if ((rc = dalloc(ctx, &ctx->outbuf, 4 * (size_t)P.nx * P.ny * P.nz))) return rc;
    if ((rc = dalloc(ctx, &ctx->ctl, 1))) return rc;
    if ((rc = dalloc(ctx, &ctx->slots, 64 * kSpread))) return rc;
    if ((rc = dalloc(ctx, &ctx->divslot, 1))) return rc;
    if ((rc = dalloc(ctx, &ctx->bar, 1))) return rc;
    if ((rc = dalloc(ctx, &ctx->ring, 4))) return rc;
    {
        int v = 0;
        CK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, P.device));
        ctx->sm_count = v;
        CK(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, P.device));
        ctx->smem_optin = (size_t)v;
        // blocks of the row kernels the SMs hold at once (their grids stop there)
        int a = 1, b = 1;
        if (P.precision == NTCFD_MIXED) {
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_sweep_rows<float, kSweepNT>, kSweepNT, 0));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_defect_rows<float, kSweepNT>, kSweepNT, 0));
        } else {
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_defect_rows<double, kSweepNT>, kSweepNT, 0));
        }
        ctx->row_resident = std::max(1, a) * ctx->sm_count;
        ctx->defect_resident = std::max(1, b) * ctx->sm_count;
        int c = 1;
        if (P.precision == NTCFD_MIXED)
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_predictor32, kP32NT, p32_smem(P.nz)));
        ctx->p32_resident = std::max(1, c) * ctx->sm_count;
    }
    if ((rc = dalloc(ctx, &ctx->coordbuf, (size_t)(P.ny + 5) + (P.nz + 5) + 8))) return rc;
    ctx->coordY = ctx->coordbuf + 1;                  // Y[j] valid for j = -1..ny+3
    ctx->coordZ = ctx->coordbuf + (P.ny + 5) + 4 + 1;
    if (ctx->csweeps > 64) return fail(ctx, NTCFD_EINVAL, "check_every must be <= 64");
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

void ntcfd_destroy(ntcfd_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaSetDevice(ctx->prm.device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    drop_graphs(ctx);
    for (void* q : ctx->allocs) cudaFree(q);
    if (ctx->dyn_trig) cudaFree(ctx->dyn_trig);
    if (ctx->dyn_buf) cudaFree(ctx->dyn_buf);
    if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
    if (ctx->rec) cudaFree(ctx->rec);
    if (ctx->rec_host) cudaFreeHost(ctx->rec_host);
    if (ctx->adj_buf) cudaFree(ctx->adj_buf);
    if (ctx->out_stream) cudaStreamSynchronize(ctx->out_stream);
    if (ctx->out_host) cudaFreeHost(ctx->out_host);
    if (ctx->out_ready) cudaEventDestroy(ctx->out_ready);
    if (ctx->out_done) cudaEventDestroy(ctx->out_done);
    if (ctx->out_stream) cudaStreamDestroy(ctx->out_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* ntcfd_last_error(const ntcfd_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

double ntcfd_time(const ntcfd_ctx* ctx) { return ctx ? ctx->time : 0.0; }

int ntcfd_set_metrics(ntcfd_ctx* ctx, const double* iDx, const double* Dxs, const double* iDy,
                      const double* Dys, const double* iDz, const double* Dzs) {
    DEV();
    if (!iDx || !Dxs || !iDy || !Dys || !iDz || !Dzs) return fail(ctx, NTCFD_EINVAL, "null metric array");
    Geom& g = ctx->g;
    const int n[3] = {g.nx, g.ny, g.nz};
    const double* iD[3] = {iDx, iDy, iDz};
    const double* Ds[3] = {Dxs, Dys, Dzs};
    for (int ax = 0; ax < 3; ++ax)
        for (int i = 0; i < n[ax] + 4; ++i)
            if (!(iD[ax][i] > 0) || !(Ds[ax][i] > 0))
                return fail(ctx, NTCFD_EINVAL, "metric %d index %d is not positive", ax, i - 1);
    // double tables: iD, Ds, riD, rDs (4 per axis) + cE..cB (6) + predictor tables (6 per axis)
    int L[3];
    size_t tot = 0;
    for (int ax = 0; ax < 3; ++ax) { L[ax] = n[ax] + 5; tot += (size_t)L[ax] * (4 + 2 + 6); }
    std::vector<double> hd(tot, 0.0);
    std::vector<float> hf(tot, 0.0f);
    size_t off = 0;
    std::vector<size_t> offs;
    auto take = [&](int len) { offs.push_back(off); size_t o = off; off += len; return o; };
    size_t o_iD[3], o_Ds[3], o_riD[3], o_rDs[3], o_c1[3], o_c2[3], o_tab[3];
    for (int ax = 0; ax < 3; ++ax) {
        const int Lx = L[ax];
        o_iD[ax] = take(Lx); o_Ds[ax] = take(Lx); o_riD[ax] = take(Lx); o_rDs[ax] = take(Lx);
        o_c1[ax] = take(Lx); o_c2[ax] = take(Lx);
        o_tab[ax] = take(6 * Lx);
        for (int i = -1; i <= n[ax] + 2; ++i) {
            const double h = iD[ax][i + 1], H = Ds[ax][i + 1];
            hd[o_iD[ax] + i + 2] = h;
            hd[o_Ds[ax] + i + 2] = H;
            hd[o_riD[ax] + i + 2] = 1.0 / h;
            hd[o_rDs[ax] + i + 2] = 1.0 / H;
        }
        // SOR coefficients over the volume: c+(i) = 1/(iD(i) Ds(i)), c-(i) = 1/(iD(i) Ds(i-1))
        for (int i = 0; i <= n[ax] + 2; ++i) {
            hd[o_c1[ax] + i + 2] = 1.0 / (iD[ax][i + 1] * Ds[ax][i + 1]);
            hd[o_c2[ax] + i + 2] = 1.0 / (iD[ax][i + 1] * Ds[ax][i]);
        }
        make_axis_tables<double>(n[ax], iD[ax], Ds[ax], hd.data() + o_tab[ax], nullptr, nullptr);
    }
    for (size_t q = 0; q < tot; ++q) hf[q] = (float)hd[q];
    if (!ctx->tabd) {
        int rc;
        if ((rc = dalloc(ctx, &ctx->tabd, tot))) return rc;
        if ((rc = dalloc(ctx, &ctx->tabf, tot))) return rc;
    }
    CK(cudaMemcpyAsync(ctx->tabd, hd.data(), tot * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->tabf, hf.data(), tot * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    const double* D = ctx->tabd + 2;
    const float* F = ctx->tabf + 2;
    g.iDx = D + o_iD[0]; g.Dxs = D + o_Ds[0]; g.iDy = D + o_iD[1]; g.Dys = D + o_Ds[1];
    g.iDz = D + o_iD[2]; g.Dzs = D + o_Ds[2];
    g.riDx = D + o_riD[0]; g.rDxs = D + o_rDs[0]; g.riDy = D + o_riD[1]; g.rDys = D + o_rDs[1];
    g.riDz = D + o_riD[2]; g.rDzs = D + o_rDs[2];
    g.cE = D + o_c1[0]; g.cW = D + o_c2[0]; g.cN = D + o_c1[1]; g.cS = D + o_c2[1];
    g.cF = D + o_c1[2]; g.cB = D + o_c2[2];
    g.cEf = F + o_c1[0]; g.cWf = F + o_c2[0]; g.cNf = F + o_c1[1]; g.cSf = F + o_c2[1];
    g.cFf = F + o_c1[2]; g.cBf = F + o_c2[2];
    ctx->scd = SorCoef<double>{g.cE, g.cW, g.cN, g.cS, g.cF, g.cB};
    ctx->scf = SorCoef<float>{g.cEf, g.cWf, g.cNf, g.cSf, g.cFf, g.cBf};
    for (int ax = 0; ax < 3; ++ax) {
        const int Lx = L[ax];
        const double* tb = D + o_tab[ax];
        const float* tf = F + o_tab[ax];
        ctx->tpd.ax[ax] = AxisTabs<double>{tb, tb + Lx, tb + 2 * Lx, tb + 3 * Lx, tb + 4 * Lx, tb + 5 * Lx};
        ctx->tpf.ax[ax] = AxisTabs<float>{tf, tf + Lx, tf + 2 * Lx, tf + 3 * Lx, tf + 4 * Lx, tf + 5 * Lx};
    }
    {
        const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
        if (ctx->prm.precision == NTCFD_MIXED)
            k_make_rd<float><<<g3, b3, 0, ctx->stream>>>(g, ctx->scf, (float*)ctx->rdR, (float*)ctx->rdB);
        else
            k_make_rd<double><<<g3, b3, 0, ctx->stream>>>(g, ctx->scd, (double*)ctx->rdR, (double*)ctx->rdB);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->metrics_set = true;
    drop_graphs(ctx);
    return 0;
}

int ntcfd_set_coords(ntcfd_ctx* ctx, const double* X, const double* Y, const double* Z) {
    DEV();
    if (!Y || !Z) return fail(ctx, NTCFD_EINVAL, "null coordinate array");
    (void)X;
    const int ny = ctx->g.ny, nz = ctx->g.nz;
    CK(cudaMemcpyAsync(ctx->coordbuf, Y, (ny + 5) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->coordbuf + (ny + 5) + 4, Z, (nz + 5) * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->coords_set = true;
    return 0;
}

// Whether ETA may be nonzero (the force kernels run).  A change rebuilds the
// step graph; going to zero also clears the force-integral arrays, which the
// adjoint reads as the step's guard pattern.
static int set_mask_flag(ntcfd_ctx* ctx, bool nonzero) {
    if (nonzero == ctx->mask_nonzero) return 0;
    CK(cudaStreamSynchronize(ctx->stream));
    drop_graphs(ctx);
    if (!nonzero) {
        const size_t cols = (size_t)ctx->g.nx * ctx->g.ny;
        CK(cudaMemsetAsync(ctx->FXz, 0, cols * sizeof(double), ctx->stream));
        CK(cudaMemsetAsync(ctx->FYz, 0, cols * sizeof(double), ctx->stream));
        CK(cudaMemsetAsync(ctx->FXy, 0, ctx->g.nx * sizeof(double), ctx->stream));
        CK(cudaMemsetAsync(ctx->FYy, 0, ctx->g.nx * sizeof(double), ctx->stream));
    }
    ctx->mask_nonzero = nonzero;
    return 0;
}

// A whole halo array (-1:n+2)^3 between its contiguous Fortran form s and the
// padded natural layout d: one thread per element, i fastest; element a of an
// axis is index a - 1.
__global__ void k_halo_unpack(Geom g, const double* __restrict__ s, double* __restrict__ d) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z * blockDim.z + threadIdx.z;
    if (a >= g.nx + 4 || b >= g.ny + 4 || c >= g.nz + 4) return;
    d[nat(g, a - 1, b - 1, c - 1)] = s[a + (size_t)(g.nx + 4) * (b + (size_t)(g.ny + 4) * c)];
}
__global__ void k_halo_pack(Geom g, const double* __restrict__ d, double* __restrict__ s) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z * blockDim.z + threadIdx.z;
    if (a >= g.nx + 4 || b >= g.ny + 4 || c >= g.nz + 4) return;
    s[a + (size_t)(g.nx + 4) * (b + (size_t)(g.ny + 4) * c)] = d[nat(g, a - 1, b - 1, c - 1)];
}

// A halo array between the host (the Fortran array, contiguous) and the
// device field: one contiguous copy through the context's staging array and a
// repacking kernel on the stream (a pitched 2-D copy moves the array as
// (ny+4)(nz+4) rows of (nx+4) doubles and runs far below the link's
// bandwidth).  The staging array is made on first use.
static int copy_halo(ntcfd_ctx* ctx, double* dev, const double* host, bool to_dev) {
    const Geom& g = ctx->g;
    const size_t n = (size_t)(g.nx + 4) * (g.ny + 4) * (g.nz + 4);
    if (!ctx->stage)
        if (int rc = dalloc(ctx, &ctx->stage, n)) return rc;
    const dim3 b3(32, 4, 2), g3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2);
    if (to_dev) {
        CK(cudaMemcpyAsync(ctx->stage, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        k_halo_unpack<<<g3, b3, 0, ctx->stream>>>(g, ctx->stage, dev);
    } else {
        k_halo_pack<<<g3, b3, 0, ctx->stream>>>(g, dev, ctx->stage);
        CK(cudaMemcpyAsync((void*)host, ctx->stage, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaGetLastError());
    return 0;
}

int ntcfd_set_mask(ntcfd_ctx* ctx, const double* eta) {
    DEV();
    ctx->smooth_active = false;
    if (!eta) return fail(ctx, NTCFD_EINVAL, "null ETA");
    int rc = copy_halo(ctx, ctx->eta, eta, true);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    const size_t n = (size_t)(ctx->g.nx + 4) * (ctx->g.ny + 4) * (ctx->g.nz + 4);
    bool nz = false;
    for (size_t q = 0; q < n && !nz; ++q) nz = eta[q] != 0.0;
    return set_mask_flag(ctx, nz);
}

int ntcfd_get_mask(ntcfd_ctx* ctx, double* eta) {
    DEV();
    if (!eta) return fail(ctx, NTCFD_EINVAL, "null ETA");
    int rc = copy_halo(ctx, ctx->eta, eta, false);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int ntcfd_set_state(ntcfd_ctx* ctx, const double* u, const double* v, const double* w, const double* p) {
    DEV();
    if (!u || !v || !w || !p) return fail(ctx, NTCFD_EINVAL, "null state array");
    int rc;
    if ((rc = copy_halo(ctx, ctx->u, u, true))) return rc;
    if ((rc = copy_halo(ctx, ctx->v, v, true))) return rc;
    if ((rc = copy_halo(ctx, ctx->w, w, true))) return rc;
    if ((rc = copy_halo(ctx, ctx->p, p, true))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int ntcfd_get_state(ntcfd_ctx* ctx, double* u, double* v, double* w, double* p) {
    DEV();
    int rc;
    if (u && (rc = copy_halo(ctx, ctx->u, u, false))) return rc;
    if (v && (rc = copy_halo(ctx, ctx->v, v, false))) return rc;
    if (w && (rc = copy_halo(ctx, ctx->w, w, false))) return rc;
    if (p && (rc = copy_halo(ctx, ctx->p, p, false))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int ntcfd_apply_bc(ntcfd_ctx* ctx) {
    DEV();
    const Geom& g = ctx->g;
    BcArgs ba{};
    ba.u = ctx->u; ba.v = ctx->v; ba.w = ctx->w; ba.p = ctx->p;
    std::memcpy(ba.bc, ctx->prm.bc, sizeof ba.bc);
    std::memcpy(ba.val, ctx->prm.bc_value, sizeof ba.val);
    ba.faceW = ctx->faceW; ba.faceE = ctx->faceE; ba.faceS = ctx->faceS;
    ba.faceN = ctx->faceN; ba.faceB = ctx->faceB; ba.faceF = ctx->faceF;
    k_bc_x<<<bc_grid_x(g), dim3(32, 8), 0, ctx->stream>>>(g, ba);
    k_bc_y<<<bc_grid_y(g), dim3(32, 8), 0, ctx->stream>>>(g, ba);
    k_bc_z<<<bc_grid_z(g), dim3(32, 8), 0, ctx->stream>>>(g, ba);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int ntcfd_get_output(ntcfd_ctx* ctx, double* pre, double* uc, double* vc, double* wc) {
    DEV();
    if (!ctx->metrics_set) return fail(ctx, NTCFD_ESTATE, "metrics not set");
    const Geom& g = ctx->g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    double* o = ctx->outbuf;
    const dim3 b3(32, 4, 2);
    k_centre<<<grid3(g, b3), b3, 0, ctx->stream>>>(g, ctx->u, ctx->v, ctx->w, ctx->p, ctx->faceW,
                                                   ctx->faceE, ctx->faceS, ctx->faceN, ctx->faceB,
                                                   ctx->faceF, o, o + n, o + 2 * n, o + 3 * n);
    CK(cudaGetLastError());
    double* dst[4] = {pre, uc, vc, wc};
    for (int q = 0; q < 4; ++q)
        if (dst[q])
            CK(cudaMemcpyAsync(dst[q], o + q * n, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

}  // extern "C"

namespace {

// Limits of the allocation-free mask scratch (defined with the scratch below).
constexpr int kNaPoly = 16384;      // polygon points
constexpr int kNaCells = 262144;    // ny * nz

// Record buffer of at least nrec steps and an instantiated step graph (the
// graph is built in eager mode too: it plans the SOR path).
int prepare_steps(ntcfd_ctx* ctx, int nrec) {
    if (nrec > ctx->rec_cap) {
        // the graph holds the record pointer: grow the record buffer, then rebuild
        const int cap = std::max(nrec, 1024);
        drop_graphs(ctx);
        if (ctx->rec) cudaFree(ctx->rec);
        ctx->rec = nullptr;
        ctx->rec_cap = 0;
        CK(cudaMalloc(&ctx->rec, sizeof(StepRec) * cap));
        ctx->rec_cap = cap;
    }
    if (!ctx->exec) {
        const int rc = ctx->prm.precision == NTCFD_MIXED ? build_graph<float>(ctx) : build_graph<double>(ctx);
        if (rc) return rc;
    }
    return 0;
}

// One step on the context's stream; its record goes to rec[ctl->step].
int launch_step(ntcfd_ctx* ctx) {
    if (ctx->prm.eager)
        return ctx->prm.precision == NTCFD_MIXED ? run_step_eager<float>(ctx) : run_step_eager<double>(ctx);
    CK(cudaGraphLaunch(ctx->exec, ctx->stream));
    return 0;
}

// Advances the simulated time by one dt per record, fills `info` (may be
// NULL) and returns the worst status of the records.
int records_to_info(ntcfd_ctx* ctx, const StepRec* rec, int nsteps, ntcfd_step_info* info,
                    const double* aoa = nullptr) {
    int status = 0;
    for (int s = 0; s < nsteps; ++s) {
        ctx->time = ctx->time + ctx->prm.dt;   // main.f90:271
        if (rec[s].timeout) status = NTCFD_ETIMEOUT;
        else if (rec[s].nonfinite && status != NTCFD_ETIMEOUT) status = NTCFD_ENONFINITE;
        else if (!rec[s].converged && status == 0) status = NTCFD_NOT_CONVERGED;
        if (info) {
            ntcfd_step_info& I = info[s];
            std::memset(&I, 0, sizeof I);
            I.sor_iters = rec[s].sor_iters;
            I.converged = rec[s].converged;
            I.sor_last_change = rec[s].last_change;
            I.cDrag = rec[s].cdrag;
            I.cLift = rec[s].clift;
            I.div_max = rec[s].divmax;
            I.dc_cycles = rec[s].cycles;
            I.launches = rec[s].launches;
            I.sor_path = ctx->resident ? NTCFD_SOR_RESIDENT : NTCFD_SOR_STREAMING;
            I.aoa = aoa ? aoa[s] : 0.0;
        }
    }
    if (status == NTCFD_ETIMEOUT) fail(ctx, status, "the resident SOR kernel's grid barrier gave up waiting");
    else if (status == NTCFD_ENONFINITE) fail(ctx, status, "non-finite value in the SOR solve");
    else if (status == NTCFD_NOT_CONVERGED) fail(ctx, status, "SOR stopped at itmax in at least one step");
    return status;
}

// End of an ntcfd_step call after `ran` steps were launched: the records of
// those steps come back (into pinned memory: a pageable destination would take
// the driver's staged, synchronous copy path on every call), the device time
// of the call, the step count and the simulated time advance by `ran`.  With
// `halted` (moving-body steps on the device), the control block comes back too
// and the steps that ran are its step count; *halted says whether a tie
// stopped them.
int finish_steps(ntcfd_ctx* ctx, int ran, ntcfd_step_info* info, const double* aoa, int* halted = nullptr) {
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if (ran > ctx->rec_host_cap) {
        if (ctx->rec_host) cudaFreeHost(ctx->rec_host);
        ctx->rec_host = nullptr;
        ctx->rec_host_cap = 0;
        CK(cudaMallocHost(&ctx->rec_host, sizeof(StepRec) * std::max(ran, 1024)));
        ctx->rec_host_cap = std::max(ran, 1024);
    }
    if (halted) {
        if (!ctx->ctl_host) CK(cudaMallocHost(&ctx->ctl_host, sizeof(Ctl)));
        CK(cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (ran > 0)
        CK(cudaMemcpyAsync(ctx->rec_host, ctx->rec, sizeof(StepRec) * ran, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaEventElapsedTime(&ctx->last_ms, ctx->ev0, ctx->ev1));
    if (halted) {
        *halted = ctx->ctl_host->halt ? ctx->ctl_host->halt_ties : 0;
        ran = std::min(ran, ctx->ctl_host->step);
    }
    ctx->istep += ran;
    return records_to_info(ctx, ctx->rec_host, ran, info, aoa);
}

// The moving body's device arrays for npts polygon points (grown, never
// shrunk); the polygon goes in as the body's.
int dyn_alloc(ntcfd_ctx* ctx, const double* az, const double* ay, int npts) {
    const Geom& g = ctx->g;
    const size_t cells = (size_t)g.ny * g.nz;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    if (npts > ctx->dyn_cap) {
        CK(cudaStreamSynchronize(ctx->stream));
        drop_dyn_graph(ctx);
        if (ctx->dyn_buf) cudaFree(ctx->dyn_buf);
        ctx->dyn_buf = nullptr;
        ctx->dyn_cap = 0;
        const size_t bytes = 2 * up(2 * (size_t)npts * sizeof(double)) + up(cells * sizeof(double)) +
                             2 * up(cells * sizeof(int)) + up(8 * sizeof(int));
        CK(cudaMalloc(&ctx->dyn_buf, bytes));
        CK(cudaMemsetAsync(ctx->dyn_buf, 0, bytes, ctx->stream));
        ctx->dyn_cap = npts;
    }
    unsigned char* q = (unsigned char*)ctx->dyn_buf;
    const size_t pb = up(2 * (size_t)ctx->dyn_cap * sizeof(double));
    DynMask& m = ctx->dyn;
    m.base = (const double*)q;
    m.poly = (double*)(q + pb);
    m.eta1 = (double*)(q + 2 * pb);
    m.flags = (int*)(q + 2 * pb + up(cells * sizeof(double)));
    m.list = (int*)(q + 2 * pb + up(cells * sizeof(double)) + up(cells * sizeof(int)));
    m.meta = (int*)(q + 2 * pb + up(cells * sizeof(double)) + 2 * up(cells * sizeof(int)));
    m.trig = ctx->dyn_trig;
    m.npts = npts;
    CK(cudaMemcpyAsync((double*)m.base, az, npts * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync((double*)m.base + npts, ay, npts * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// The per-step angle table of a call of nsteps steps and, unless the context
// is eager or the graph could not be built here, the moving-body step graph.
int prepare_dyn(ntcfd_ctx* ctx, int nsteps) {
    if (nsteps > ctx->dyn_trig_cap) {
        CK(cudaStreamSynchronize(ctx->stream));
        drop_dyn_graph(ctx);
        if (ctx->dyn_trig) cudaFree(ctx->dyn_trig);
        ctx->dyn_trig = nullptr;
        ctx->dyn_trig_cap = 0;
        const int cap = std::max(nsteps, 1024);
        CK(cudaMalloc(&ctx->dyn_trig, 2 * sizeof(double) * cap));
        ctx->dyn_trig_cap = cap;
        ctx->dyn.trig = ctx->dyn_trig;
    }
    if (ctx->prm.eager || ctx->exec_dyn || !ctx->dyn_graph_err.empty()) return 0;
    const int rc = ctx->prm.precision == NTCFD_MIXED ? build_dyn_graph<float>(ctx) : build_dyn_graph<double>(ctx);
    if (rc) {
        // this device or driver does not take the graph (an IF node around the
        // step's own loops): the steps launch the mask kernels one by one instead
        ctx->dyn_graph_err = ctx->err;
        drop_dyn_graph(ctx);
        cudaGetLastError();
    }
    return 0;
}

// The mask kernels of a moving-body step launched one by one (eager contexts,
// or where the moving-body graph could not be built); *ties receives the
// step's exact vertex/grid ties.
int dyn_mask_eager(ntcfd_ctx* ctx, int* ties) {
    const Geom& g = ctx->g;
    const DynMask m = ctx->dyn;
    const int cells = g.ny * g.nz;
    cudaStream_t st = ctx->stream;
    k_dyn_rotate<512><<<1, 512, 0, st>>>(g.ny, g.nz, ctx->coordY, ctx->coordZ, m, ctx->ctl);
    k_dyn_main<<<dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), 0, st>>>(g.ny, g.nz, ctx->coordY,
                                                                              ctx->coordZ, m, ctx->ctl);
    k_dyn_points<<<(m.npts + 127) / 128, 128, 0, st>>>(g.ny, g.nz, ctx->coordY, ctx->coordZ, m, ctx->ctl);
    k_dyn_compact<<<(cells + 255) / 256, 256, 0, st>>>(cells, m, ctx->ctl);
    k_dyn_sub<256><<<2 * ctx->sm_count, 256, 0, st>>>(g.nz, ctx->coordY, ctx->coordZ, m, ctx->ctl);
    k_dyn_extrude<<<dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2), dim3(32, 4, 2), 0, st>>>(
        g, m.eta1, ctx->eta, ctx->ctl);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ties, &m.meta[5], sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace

extern "C" {

int ntcfd_step(ntcfd_ctx* ctx, int nsteps, ntcfd_step_info* info) {
    DEV();
    if (nsteps < 0) return fail(ctx, NTCFD_EINVAL, "nsteps < 0");
    if (!ctx->metrics_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_metrics must come before ntcfd_step");
    if (is_slab(ctx))
        return fail(ctx, NTCFD_EINVAL, "a z-slab context (a Back or Front wall of kind NTCFD_BC_INTERFACE) "
                    "advances through ntcfd_slab_stage");
    if (nsteps == 0) return 0;
    // a moving body in this call: its steps rebuild ETA on the device
    const bool dyn = ctx->dyn_start > 0 && ctx->istep + nsteps >= ctx->dyn_start;
    if (dyn)
        if (int rc = set_mask_flag(ctx, true)) return rc;
    if (int rc = prepare_steps(ctx, nsteps)) return rc;
    if (dyn)
        if (int rc = prepare_dyn(ctx, nsteps)) return rc;
    std::vector<double> aoa(nsteps, 0.0), trig(dyn ? 2 * (size_t)nsteps : 0, 0.0);
    double t = ctx->time;
    for (int s = 0; s < nsteps; ++s) {
        const long long istep = ctx->istep + s + 1;
        if (dyn && istep >= ctx->dyn_start) {
            // dynamic_AOA (airfoil.f90:313-317): PI is the default-real literal 3.14159265359
            const double PI = (double)3.14159265359f;
            const double frequency = ctx->dyn_rf / PI;
            aoa[s] = ctx->dyn_aoa1 +
                     10 * std::fabs(std::sin(2 * PI * frequency * (t - ctx->prm.dt * (double)(ctx->dyn_start - 1))));
            // the rotation of airfoil.f90:597-611 (pi = 4 atan(1) there)
            const double pr = 4.0 * std::atan(1.0);
            trig[2 * s] = std::cos((-aoa[s]) * pr / 180);
            trig[2 * s + 1] = std::sin((-aoa[s]) * pr / 180);
        }
        t = t + ctx->prm.dt;
    }
    if (dyn) CK(cudaMemcpyAsync(ctx->dyn_trig, trig.data(), trig.size() * sizeof(double), cudaMemcpyHostToDevice,
                                ctx->stream));
    CK(cudaMemsetAsync(&ctx->ctl->step, 0, sizeof(int), ctx->stream));
    CK(cudaMemsetAsync(&ctx->ctl->halt, 0, 2 * sizeof(int), ctx->stream));
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    const bool graph_dyn = dyn && ctx->exec_dyn;
    for (int s = 0; s < nsteps; ++s) {
        if (dyn && ctx->istep + s + 1 >= ctx->dyn_start) {
            if (graph_dyn) {
                CK(cudaGraphLaunch(ctx->exec_dyn, ctx->stream));
                continue;
            }
            int ties = 0;
            if (int rc = dyn_mask_eager(ctx, &ties)) return rc;
            if (ties) {
                // steps 0..s-1 ran: account for them (time, step count, records) before
                // returning, so that the host's view matches the device state
                if (int r2 = finish_steps(ctx, s, info, aoa.data())) return r2;
                return fail(ctx, NTCFD_EINVAL, "step %d of this call (%d ran): %d exact vertex/grid ties: the "
                            "reference resolves them by moving the grid", s + 1, s, ties);
            }
        }
        if (int rc = launch_step(ctx)) return rc;
    }
    if (!graph_dyn) return finish_steps(ctx, nsteps, info, aoa.data());
    int halted = 0;
    const long long before = ctx->istep;
    const int rc = finish_steps(ctx, nsteps, info, aoa.data(), &halted);
    if (halted) {
        const int ran = (int)(ctx->istep - before);
        if (rc == 0 || rc == NTCFD_NOT_CONVERGED)
            return fail(ctx, NTCFD_EINVAL, "step %d of this call (%d ran): %d exact vertex/grid ties: the "
                        "reference resolves them by moving the grid", ran + 1, ran, halted);
    }
    return rc;
}

// ------------------------------------------------------------ z-slabs
// One process (one GPU) per slab of z planes (Mpi_division.f90:6-24); the
// caller exchanges the planes between stages as main.f90:163-201,220-240 and
// GS.f90:20-28 do and takes the max of the sweep changes over the slabs
// (GS.f90:70).  The stages launch the same kernels as a step of the FP64
// streaming path, so a decomposed solve repeats the single-domain one bit for
// bit when the exchanges deliver the neighbours' planes.

static double* slab_field(ntcfd_ctx* ctx, int field, long long* plane) {
    const Geom& g = ctx->g;
    *plane = g.pz;
    switch (field) {
        case NTCFD_FIELD_U: return ctx->u;
        case NTCFD_FIELD_V: return ctx->v;
        case NTCFD_FIELD_W: return ctx->w;
        case NTCFD_FIELD_P: return ctx->p;
        case NTCFD_FIELD_WSTAR: return ctx->ws;
        case NTCFD_FIELD_E_RED: *plane = g.mz; return (double*)ctx->eR;
        case NTCFD_FIELD_E_BLACK: *plane = g.mz; return (double*)ctx->eB;
        default: return nullptr;
    }
}

long long ntcfd_slab_plane_elems(const ntcfd_ctx* ctx, int field) {
    if (!ctx || field < NTCFD_FIELD_U || field > NTCFD_FIELD_E_BLACK) return -1;
    return field >= NTCFD_FIELD_E_RED ? ctx->g.mz : ctx->g.pz;
}

int ntcfd_slab_planes(ntcfd_ctx* ctx, int field, int k0, int count, double* buf, int put) {
    DEV();
    long long plane = 0;
    double* f = slab_field(ctx, field, &plane);
    if (!f) return fail(ctx, NTCFD_EINVAL, "unknown field %d", field);
    if (ctx->prm.precision != NTCFD_FP64) return fail(ctx, NTCFD_EINVAL, "the z-slab stages run in FP64");
    if (!buf || count < 1 || k0 < -1 || k0 + count - 1 > ctx->g.nz + 2)
        return fail(ctx, NTCFD_EINVAL, "planes %d..%d outside -1..nz+2", k0, k0 + count - 1);
    double* dev = f + plane * (long long)(k0 + 1);
    const size_t bytes = sizeof(double) * (size_t)plane * count;
    if (put) CK(cudaMemcpyAsync(dev, buf, bytes, cudaMemcpyDefault, ctx->stream));
    else CK(cudaMemcpyAsync(buf, dev, bytes, cudaMemcpyDefault, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int ntcfd_slab_stage(ntcfd_ctx* ctx, int stage, int colour) {
    DEV();
    if (!ctx->metrics_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_metrics must come first");
    if (ctx->prm.precision != NTCFD_FP64) return fail(ctx, NTCFD_EINVAL, "the z-slab stages run in FP64");
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    cudaStream_t st = ctx->stream;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    double *eR = (double*)ctx->eR, *eB = (double*)ctx->eB, *dR = (double*)ctx->dR, *dB = (double*)ctx->dB;
    switch (stage) {
        case NTCFD_STAGE_PREDICT:   // [Smagorinsky] + predictor: u, v, w with two halo planes
            // the reference-aliased Smagorinsky reads storage offsets of the whole
            // domain's arrays (smagorinsky.f90 with the arrays' declared shape), which a
            // slab does not hold
            if (is_slab(ctx) && P.LES && P.smag_mode == NTCFD_SMAG_REF_ALIASED)
                return fail(ctx, NTCFD_EINVAL, "z-slabs take LES with smag_mode = NTCFD_SMAG_STAGGERED");
            launch_predictor(ctx, st);
            break;
        case NTCFD_STAGE_RHS:       // rhs, the solve's defect and e = 0: w* and p with one halo plane
            k_rhs<<<walk_grid(g, ctx->sm_count), walk_block(), 0, st>>>(g, ctx->scd, ctx->u, ctx->v, ctx->w,
                                                                        ctx->us, ctx->vs, ctx->ws, ctx->b, P.dt, back_iface(ctx));
            k_sor_begin<<<1, 1, 0, st>>>(ctx->ctl, P.itmax, 0, 0);
            k_defect<double><<<g3, b3, 0, st>>>(g, ctx->scd, ctx->p, ctx->b, dR, dB, eR, eB,
                                                (const double*)ctx->rdR, (const double*)ctx->rdB, ctx->ctl, 0, 0,
                                                nullptr, nullptr, 0, 0);
            k_clear_e<double><<<g3, b3, 0, st>>>(g, eR, eB);
            // the ghost planes of e hold the neighbours' last planes of the previous
            // solve: theirs start from zero too
            for (double* e : {eR, eB}) {
                CK(cudaMemsetAsync(e, 0, sizeof(double) * g.mz * 2, st));
                CK(cudaMemsetAsync(e + g.mz * (g.nz + 2), 0, sizeof(double) * g.mz * 2, st));
            }
            CK(cudaMemsetAsync(ctx->slots, 0, sizeof(unsigned long long) * kSpread, st));
            break;
        case NTCFD_STAGE_HALFSWEEP: {   // colour 0: (i+j+k) even in the slab's own k; e of the other colour
            if (colour != 0 && colour != 1) return fail(ctx, NTCFD_EINVAL, "colour must be 0 or 1");
            const dim3 bs = Sweep<double>::block(), gs = Sweep<double>::grid(g, ctx->row_resident);
            Sweep<double>::fn<<<gs, bs, 0, st>>>(g, ctx->scd, colour ? eB : eR, colour ? eR : eB,
                                                 colour ? dB : dR, (const double*)(colour ? ctx->rdB : ctx->rdR),
                                                 colour, P.omega, ctx->ctl, 0, P.itmax, P.itmax, 0, ctx->slots, 0);
            break;
        }
        case NTCFD_STAGE_CORRECT:   // p += e
            k_correct<double><<<g3, b3, 0, st>>>(g, ctx->p, eR, eB);
            break;
        case NTCFD_STAGE_PROJECT: { // projection, forcing, velocity commit, BCs on the physical faces
            ProjArgs pj{ctx->u, ctx->v, ctx->w, ctx->us, ctx->vs, ctx->ws, ctx->p, ctx->eta, ctx->partZ,
                        ctx->partY, P.dt, P.u_solid[0], P.u_solid[1], P.u_solid[2], kProjKc};
            k_project<<<dim3((g.nx + 31) / 32, (g.ny + 3) / 4, ctx->nchunk), dim3(32, 4, 1), 0, st>>>(g, pj);
            BcArgs ba{};
            ba.u = ctx->u; ba.v = ctx->v; ba.w = ctx->w; ba.p = ctx->p;
            std::memcpy(ba.bc, P.bc, sizeof ba.bc);
            std::memcpy(ba.val, P.bc_value, sizeof ba.val);
            ba.faceW = ctx->faceW; ba.faceE = ctx->faceE; ba.faceS = ctx->faceS;
            ba.faceN = ctx->faceN; ba.faceB = ctx->faceB; ba.faceF = ctx->faceF;
            k_bc_x<<<bc_grid_x(g), dim3(32, 8), 0, st>>>(g, ba);
            k_bc_y<<<bc_grid_y(g), dim3(32, 8), 0, st>>>(g, ba);
            k_bc_z<<<bc_grid_z(g), dim3(32, 8), 0, st>>>(g, ba);
            ctx->time = ctx->time + P.dt;
            ctx->istep += 1;
            break;
        }
        default:
            return fail(ctx, NTCFD_EINVAL, "unknown stage %d", stage);
    }
    CK(cudaGetLastError());
    return 0;
}

int ntcfd_slab_change(ntcfd_ctx* ctx, double* max_change) {
    DEV();
    if (!max_change) return fail(ctx, NTCFD_EINVAL, "null max_change");
    unsigned long long h[kSpread];
    CK(cudaMemcpyAsync(h, ctx->slots, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->slots, 0, sizeof h, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long m = 0;
    for (int q = 0; q < kSpread; ++q) m = h[q] > m ? h[q] : m;
    std::memcpy(max_change, &m, sizeof m);   // |change| as its bit pattern; NaN stays NaN
    return 0;
}

int ntcfd_output_async(ntcfd_ctx* ctx, double* pre, double* uc, double* vc, double* wc) {
    DEV();
    if (!ctx->metrics_set) return fail(ctx, NTCFD_ESTATE, "metrics not set");
    const Geom& g = ctx->g;
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    if (ctx->out_pending) {   // one output in flight: its buffers are reused
        CK(cudaEventSynchronize(ctx->out_done));
        ctx->out_pending = false;
    }
    double* dst[4] = {pre, uc, vc, wc};
    bool staged[4] = {false, false, false, false}, any_staged = false;
    for (int q = 0; q < 4; ++q) {
        if (!dst[q]) continue;
        staged[q] = !dma_reachable(dst[q]);
        any_staged |= staged[q];
    }
    if (!ctx->out_dev) {
        double* q = nullptr;
        if (int rc = dalloc(ctx, &q, 4 * n)) return rc;
        ctx->out_dev = q;
        CK(cudaStreamCreateWithFlags(&ctx->out_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->out_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->out_done, cudaEventDisableTiming));
    }
    if (any_staged && !ctx->out_host) CK(cudaMallocHost(&ctx->out_host, 4 * n * sizeof(double)));
    double* o = ctx->out_dev;
    const dim3 b3(32, 4, 2);
    k_centre<<<grid3(g, b3), b3, 0, ctx->stream>>>(g, ctx->u, ctx->v, ctx->w, ctx->p, ctx->faceW,
                                                   ctx->faceE, ctx->faceS, ctx->faceN, ctx->faceB,
                                                   ctx->faceF, o, o + n, o + 2 * n, o + 3 * n);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->out_ready, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->out_stream, ctx->out_ready, 0));
    for (int q = 0; q < 4; ++q) {
        ctx->out_dst[q] = dst[q];
        ctx->out_staged[q] = staged[q];
        if (!dst[q]) continue;
        double* to = staged[q] ? ctx->out_host + q * n : dst[q];
        CK(cudaMemcpyAsync(to, o + q * n, n * sizeof(double), cudaMemcpyDefault, ctx->out_stream));
    }
    ctx->out_n = n;
    if (any_staged) CK(cudaLaunchHostFunc(ctx->out_stream, scatter_output, ctx));
    CK(cudaEventRecord(ctx->out_done, ctx->out_stream));
    ctx->out_pending = true;
    return 0;
}

int ntcfd_output_wait(ntcfd_ctx* ctx) {
    DEV();
    if (!ctx->out_pending) return fail(ctx, NTCFD_ESTATE, "no ntcfd_output_async in flight");
    CK(cudaEventSynchronize(ctx->out_done));
    ctx->out_pending = false;
    return 0;
}

int ntcfd_set_dynamic_aoa(ntcfd_ctx* ctx, const double* az, const double* ay, int npts, double aoa1,
                          double reduce_frequency, double zc, double yc, int start_step) {
    DEV();
    if (npts == 0) {
        ctx->dyn_start = 0;
        CK(cudaStreamSynchronize(ctx->stream));
        drop_dyn_graph(ctx);
        return 0;
    }
    if (!az || !ay || npts < 3) return fail(ctx, NTCFD_EINVAL, "polygon needs >= 3 points");
    if (start_step < 1) return fail(ctx, NTCFD_EINVAL, "start_step must be >= 1");
    if (!std::isfinite(aoa1) || !std::isfinite(reduce_frequency) || !std::isfinite(zc) || !std::isfinite(yc))
        return fail(ctx, NTCFD_EINVAL, "non-finite dynamic angle parameters");
    if (!ctx->coords_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_coords must come first");
    ctx->smooth_active = false;
    CK(cudaStreamSynchronize(ctx->stream));
    drop_dyn_graph(ctx);     // the graph holds the polygon's size and centre
    if (int rc = dyn_alloc(ctx, az, ay, npts)) return rc;
    ctx->dyn.zc = zc;
    ctx->dyn.yc = yc;
    ctx->dyn_aoa1 = aoa1;
    ctx->dyn_rf = reduce_frequency;
    ctx->dyn_start = start_step;
    return 0;
}

int ntcfd_last_step_ms(const ntcfd_ctx* ctx, float* ms) {
    if (!ctx || !ms) return NTCFD_EINVAL;
    *ms = ctx->last_ms;
    return 0;
}

int ntcfd_time_kernels(ntcfd_ctx* ctx, int reps, ntcfd_kernel_times* out) {
    DEV();
    if (!out || reps < 1) return fail(ctx, NTCFD_EINVAL, "bad arguments");
    if (!ctx->metrics_set) return fail(ctx, NTCFD_ESTATE, "metrics not set");
    std::memset(out, 0, sizeof *out);
    return ctx->prm.precision == NTCFD_MIXED ? time_kernels_t<float>(ctx, reps, out)
                                            : time_kernels_t<double>(ctx, reps, out);
}

// ------------------------------------------------------------------ masks
int ntcfd_build_mask_cylinder(ntcfd_ctx* ctx, double zc, double yc, double r) {
    DEV();
    ctx->smooth_active = false;
    if (!ctx->metrics_set || !ctx->coords_set) return fail(ctx, NTCFD_ESTATE, "metrics and coordinates first");
    if (int rc = set_mask_flag(ctx, true)) return rc;
    const Geom& g = ctx->g;
    double* eta1 = ctx->outbuf;  // scratch: nz*ny
    k_cylinder<<<dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), 0, ctx->stream>>>(
        g.ny, g.nz, ctx->coordY, ctx->coordZ, g.iDx, g.iDy, g.iDz, zc, yc, r, eta1);
    const dim3 b3(32, 4, 2);
    k_extrude<<<dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2), b3, 0, ctx->stream>>>(
        g, eta1, ctx->eta);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int ntcfd_build_mask_smooth(ntcfd_ctx* ctx, const double* az_in, const double* ay_in, int npts, double aoa,
                            double zc, double yc, double width) {
    DEV();
    ctx->smooth_active = false;
    if (!az_in || !ay_in || npts < 3) return fail(ctx, NTCFD_EINVAL, "polygon needs >= 3 points");
    if (!(width > 0) || !std::isfinite(aoa) || !std::isfinite(zc) || !std::isfinite(yc))
        return fail(ctx, NTCFD_EINVAL, "width must be positive, the angle and centre finite");
    if (!ctx->coords_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_coords must come first");
    if (int rc = set_mask_flag(ctx, true)) return rc;
    const Geom& g = ctx->g;
    const size_t cells = (size_t)g.ny * g.nz;
    // the vertices moved as ntcfd_build_mask_polygon moves them (airfoil.f90:597-611), and
    // their derivatives with respect to the angle in radians (phi = -angle):
    //   z1 = c z0 - s y0, y1 = s z1 + c y0 (the new z1: the reference's order)
    std::vector<double> h(4 * (size_t)npts);
    const double PI = 4.0 * std::atan(1.0);
    const double c = std::cos((-aoa) * PI / 180), sn = std::sin((-aoa) * PI / 180);
    for (int i = 0; i < npts; ++i) {
        const double z0 = az_in[i] - 0.25, y0 = ay_in[i];
        const double z1 = c * z0 - sn * y0;
        const double y1 = sn * z1 + c * y0;
        const double dz1 = -sn * z0 - c * y0;            // d/dphi
        const double dy1 = c * z1 + sn * dz1 - sn * y0;
        h[i] = z1 + zc + 0.25;
        h[npts + i] = y1 + yc;
        h[2 * npts + i] = -dz1;                          // d/dangle = -d/dphi
        h[3 * npts + i] = -dy1;
    }
    if (!ctx->deta_daoa) {
        double* q = nullptr;
        if (int rc = dalloc(ctx, &q, cells)) return rc;
        ctx->deta_daoa = q;
    }
    double* dp = nullptr;
    CK(cudaMalloc(&dp, sizeof(double) * 4 * npts));
    CK(cudaMemcpyAsync(dp, h.data(), sizeof(double) * 4 * npts, cudaMemcpyHostToDevice, ctx->stream));
    double* eta1 = ctx->outbuf;
    k_smooth_mask<<<dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), 0, ctx->stream>>>(
        g.ny, g.nz, ctx->coordY, ctx->coordZ, dp, dp + npts, dp + 2 * npts, dp + 3 * npts, npts, width, eta1,
        ctx->deta_daoa);
    const dim3 b3(32, 4, 2);
    k_extrude<<<dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2), b3, 0, ctx->stream>>>(
        g, eta1, ctx->eta);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(dp);
    ctx->smooth_active = true;
    return 0;
}

int ntcfd_build_mask_polygon(ntcfd_ctx* ctx, const double* az_in, const double* ay_in, int npts,
                             double aoa, double zc, double yc, int* ties_out) {
    DEV();
    ctx->smooth_active = false;
    if (!az_in || !ay_in || npts < 3) return fail(ctx, NTCFD_EINVAL, "polygon needs >= 3 points");
    if (!ctx->coords_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_coords must come first");
    if (int rc = set_mask_flag(ctx, true)) return rc;
    const Geom& g = ctx->g;
    // airfoil.f90:597-611 on the host: shift by the quarter chord, rotate by
    // -AOA (ay uses the already rotated az, as in the reference), translate.
    std::vector<double> az(az_in, az_in + npts), ay(ay_in, ay_in + npts);
    const double PI = 4.0 * std::atan(1.0);
    for (int i = 0; i < npts; ++i) {
        az[i] = az[i] - 0.25;
        az[i] = std::cos((-aoa) * PI / 180) * az[i] - std::sin((-aoa) * PI / 180) * ay[i];
        ay[i] = std::sin((-aoa) * PI / 180) * az[i] + std::cos((-aoa) * PI / 180) * ay[i];
        az[i] = az[i] + zc;
        ay[i] = ay[i] + yc;
        az[i] = az[i] + 0.25;
    }
    // node coordinates back on the host for the A, B, C, E search (airfoil.f90:615-654)
    std::vector<double> Y(g.ny + 5), Z(g.nz + 5);
    CK(cudaMemcpyAsync(Y.data(), ctx->coordbuf, (g.ny + 5) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Z.data(), ctx->coordbuf + (g.ny + 5) + 4, (g.nz + 5) * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    auto Yf = [&](int j) { return Y[j + 1]; };
    auto Zf = [&](int k) { return Z[k + 1]; };
    double miny = ay[0], maxy = ay[0], minz = az[0], maxz = az[0];
    for (int i = 1; i < npts; ++i) {
        miny = std::min(miny, ay[i]); maxy = std::max(maxy, ay[i]);
        minz = std::min(minz, az[i]); maxz = std::max(maxz, az[i]);
    }
    int A = 0, B = 0, C = 0, E = 0;
    for (int j = 1; j <= g.ny; ++j) if (Yf(j) > miny) { A = j - 1; break; }
    for (int j = 1; j <= g.ny; ++j) if (Yf(j) > maxy) { B = j; break; }
    for (int k = 1; k <= g.nz; ++k) if (Zf(k) > minz) { C = k - 1; break; }
    for (int k = 1; k <= g.nz; ++k) if (Zf(k) > maxz) { E = k; break; }
    // device work buffers
    double* daz = nullptr;
    int* dint = nullptr;
    const size_t cells = (size_t)g.ny * g.nz;
    CK(cudaMalloc(&daz, sizeof(double) * 2 * npts));
    CK(cudaMalloc(&dint, sizeof(int) * (2 * cells + 1)));
    double* day = daz + npts;
    int* points = dint;
    int* list = dint + cells;
    int* ties = dint + 2 * cells;
    CK(cudaMemcpyAsync(daz, az.data(), sizeof(double) * npts, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(day, ay.data(), sizeof(double) * npts, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(dint, 0, sizeof(int) * (2 * cells + 1), ctx->stream));
    double* eta1 = ctx->outbuf;
    k_ray_main<<<dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), 0, ctx->stream>>>(
        g.ny, g.nz, ctx->coordY, ctx->coordZ, daz, day, npts, eta1, ties);
    k_ray_points<<<(npts + 127) / 128, 128, 0, ctx->stream>>>(g.ny, g.nz, ctx->coordY, ctx->coordZ, daz,
                                                                day, npts, A, B, C, E, points);
    std::vector<int> hp(cells);
    CK(cudaMemcpyAsync(hp.data(), points, sizeof(int) * cells, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<int> hl;
    for (size_t q = 0; q < cells; ++q)
        if (hp[q]) hl.push_back((int)q);
    if (!hl.empty()) {
        CK(cudaMemcpyAsync(list, hl.data(), sizeof(int) * hl.size(), cudaMemcpyHostToDevice, ctx->stream));
        k_ray_sub<256><<<(unsigned)hl.size(), 256, 0, ctx->stream>>>(g.nz, ctx->coordY, ctx->coordZ, daz,
                                                                    day, npts, list, eta1, ties);
    }
    const dim3 b3(32, 4, 2);
    k_extrude<<<dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2), b3, 0, ctx->stream>>>(
        g, eta1, ctx->eta);
    int hties = 0;
    CK(cudaMemcpyAsync(&hties, ties, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(daz);
    cudaFree(dint);
    if (ties_out) *ties_out = hties;
    if (hties)
        return fail(ctx, NTCFD_EINVAL,
                    "%d exact vertex/grid ties: the reference resolves them by moving the grid", hties);
    return 0;
}

// ------------------------------------------- ray casting without allocation
}  // extern "C"

// Scratch of ntcfd_build_mask_polygon_noalloc: one fixed device array per
// device that loads the library.  Layout (every offset a multiple of 256 B):
// the body polygon az[npts], ay[npts] (room for kNaPoly points each, double),
// the moved polygon (the same), the cut-cell flags and the compacted cut-cell
// list (kNaCells int each), then the bounds A, B, C, E, the listed-cell count
// and the tie counter (int), the rotation's cosine and sine (double) and a
// control block whose step index and halt flag the mask kernels read.
namespace {
constexpr size_t kNaPolyOff = 2 * sizeof(double) * (size_t)kNaPoly;
constexpr size_t kNaFlagsOff = 2 * kNaPolyOff;
constexpr size_t kNaListOff = kNaFlagsOff + sizeof(int) * (size_t)kNaCells;
constexpr size_t kNaMetaOff = kNaListOff + sizeof(int) * (size_t)kNaCells;
constexpr size_t kNaTrigOff = kNaMetaOff + 64;
constexpr size_t kNaCtlOff = kNaMetaOff + 256;
constexpr size_t kNaBytes = kNaCtlOff + 256;   // 2.5 MiB + 512 B
static_assert(sizeof(Ctl) <= 256, "control block outgrew its scratch slot");
}  // namespace

static __device__ __align__(256) unsigned char g_mask_scratch[kNaBytes];

namespace {
std::mutex g_na_mu;
void* g_na_addr[256] = {};

// Device address of g_mask_scratch on the current device (the context's),
// looked up once per device: in host code the symbol is only a stand-in.
int noalloc_scratch(ntcfd_ctx* ctx, unsigned char** out) {
    const int dev = ctx->prm.device;
    if (dev < 0 || dev >= 256) return fail(ctx, NTCFD_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_addr[dev]) {
        void* a = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&a, g_mask_scratch);
        if (e != cudaSuccess || !a)
            return fail(ctx, NTCFD_ECUDA, "cudaGetSymbolAddress(g_mask_scratch) failed: %s",
                        cudaGetErrorString(e));
        g_na_addr[dev] = a;
    }
    *out = (unsigned char*)g_na_addr[dev];
    return 0;
}
}  // namespace

// The whole ray casting runs on the device, as a moving body's mask does
// (k_dyn_*): the polygon is turned and its bounds found on the device, the
// cut cells are compacted there with an atomic counter, and the host reads
// back only the tie count at the end, so the call makes one stream
// synchronisation and no host-side copy of coordinates or flags.
extern "C" int ntcfd_build_mask_polygon_noalloc(ntcfd_ctx* ctx, const double* az_in, const double* ay_in,
                                                int npts, double aoa, double zc, double yc, int* ties_out) {
    DEV();
    ctx->smooth_active = false;
    if (!az_in || !ay_in || npts < 3) return fail(ctx, NTCFD_EINVAL, "polygon needs >= 3 points");
    if (!ctx->coords_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_coords must come first");
    const Geom& g = ctx->g;
    const size_t cells = (size_t)g.ny * g.nz;
    if (npts > kNaPoly)
        return fail(ctx, NTCFD_EINVAL, "polygon has %d points; the allocation-free variant takes at most %d",
                    npts, kNaPoly);
    if (cells > (size_t)kNaCells)
        return fail(ctx, NTCFD_EINVAL, "ny*nz = %zu cells; the allocation-free variant takes at most %d",
                    cells, kNaCells);
    if (int rc = set_mask_flag(ctx, true)) return rc;
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch(ctx, &base)) return rc;
    DynMask m{};
    m.base = reinterpret_cast<const double*>(base);
    m.poly = reinterpret_cast<double*>(base + kNaPolyOff);
    m.flags = reinterpret_cast<int*>(base + kNaFlagsOff);
    m.list = reinterpret_cast<int*>(base + kNaListOff);
    m.meta = reinterpret_cast<int*>(base + kNaMetaOff);
    m.trig = reinterpret_cast<const double*>(base + kNaTrigOff);
    m.npts = npts;
    m.zc = zc;
    m.yc = yc;
    m.eta1 = ctx->outbuf;
    Ctl* ctl = reinterpret_cast<Ctl*>(base + kNaCtlOff);
    // the rotation of airfoil.f90:597-611 (pi = 4 atan(1) there); the array keeps
    // the previous call's contents, so the control block (step 0, no halt) is
    // cleared here and the counters by k_dyn_rotate, the flags by k_dyn_main
    const double PI = 4.0 * std::atan(1.0);
    const double trig[2] = {std::cos((-aoa) * PI / 180), std::sin((-aoa) * PI / 180)};
    cudaStream_t st = ctx->stream;
    CK(cudaMemsetAsync(ctl, 0, sizeof(Ctl), st));
    CK(cudaMemcpyAsync((double*)m.trig, trig, sizeof trig, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((double*)m.base, az_in, sizeof(double) * npts, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync((double*)m.base + npts, ay_in, sizeof(double) * npts, cudaMemcpyHostToDevice, st));
    k_dyn_rotate<512><<<1, 512, 0, st>>>(g.ny, g.nz, ctx->coordY, ctx->coordZ, m, ctl);
    k_dyn_main<<<dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), 0, st>>>(g.ny, g.nz, ctx->coordY,
                                                                              ctx->coordZ, m, ctl);
    k_dyn_points<<<(npts + 127) / 128, 128, 0, st>>>(g.ny, g.nz, ctx->coordY, ctx->coordZ, m, ctl);
    k_dyn_compact<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>((int)cells, m, ctl);
    k_dyn_sub<256><<<2 * ctx->sm_count, 256, 0, st>>>(g.nz, ctx->coordY, ctx->coordZ, m, ctl);
    k_dyn_extrude<<<dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 3) / 4, (g.nz + 4 + 1) / 2), dim3(32, 4, 2), 0, st>>>(
        g, m.eta1, ctx->eta, ctl);
    CK(cudaGetLastError());
    int hties = 0;
    CK(cudaMemcpyAsync(&hties, &m.meta[5], sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (ties_out) *ties_out = hties;
    if (hties)
        return fail(ctx, NTCFD_EINVAL,
                    "%d exact vertex/grid ties: the reference resolves them by moving the grid", hties);
    return 0;
}

// ============================================================ body force
extern "C" int ntcfd_set_body_force(ntcfd_ctx* ctx, const double* fu, const double* fv, const double* fw) {
    DEV();
    const Geom& g = ctx->g;
    const size_t N = ctx->nat_elems;
    if (!fu && !fv && !fw) {
        if (ctx->fb) {
            // the graph holds the pointer: drop it so that the next step rebuilds without the force
            CK(cudaStreamSynchronize(ctx->stream));
            drop_graphs(ctx);
            ctx->fb = nullptr;   // the storage stays in ctx->allocs
        }
        return 0;
    }
    if (!ctx->fb) {
        double* q = nullptr;
        if (int rc = dalloc(ctx, &q, 3 * N)) return rc;
        ctx->fb = q;
        drop_graphs(ctx);
    }
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    const double* src[3] = {fu, fv, fw};
    const dim3 b3(32, 4, 2);
    for (int c = 0; c < 3; ++c) {
        double* dst = ctx->fb + c * N;
        if (!src[c]) {
            CK(cudaMemsetAsync(dst, 0, N * sizeof(double), ctx->stream));
            continue;
        }
        for (size_t q = 0; q < n; ++q)
            if (!std::isfinite(src[c][q])) return fail(ctx, NTCFD_EINVAL, "non-finite body force");
        CK(cudaMemcpyAsync(ctx->outbuf, src[c], n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        k_interior_in<<<grid3(g, b3), b3, 0, ctx->stream>>>(g, ctx->outbuf, dst);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

// ============================================================ adjoint
namespace {

// Workspace of ntcfd_adjoint: one device buffer kept in the context and
// grown when a call needs more, carved into 256-byte aligned pieces.
struct AdjCarve {
    size_t off = 0;
    char* base = nullptr;   // null while sizing
    template <class T>
    void take(T** out, size_t n) {
        off = (off + 255) & ~size_t(255);
        *out = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += n * sizeof(T);
    }
};

struct AdjBufs {
    double *lu, *lv, *lw, *lp, *lpn, *lus, *lvs, *lws, *z, *zprev, *badj, *lb, *wD, *wL, *lnut, *gf, *gval;
    double *geta, *etacol;       // dJ/dETA summed over the steps, its column sums (smoothed mask only)
    unsigned long long* slot;
    int solves;                  // adjoint solves done (the guess extrapolates after two)
    cudaEvent_t e0, e1;          // around each solve
    double solve_ms;
};

// Reverse of one step: on entry lu, lv, lw, lp hold the adjoint of the state
// after the step; on return the adjoint of the state before it.  (su, sv, sw)
// is the velocity before the step, `guards` the step's force-integral guards;
// with A.geta, po and pn are the pressure before and after the step.
template <class Tc>
int adjoint_step(ntcfd_ctx* ctx, AdjBufs& A, const double* su, const double* sv, const double* sw,
                 const double* po, const double* pn, const unsigned char* guards, double scaleD, double scaleL,
                 double zeta_rel, int itmax, double omega, long long* sweeps, int* unconverged) {
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    cudaStream_t st = ctx->stream;
    const size_t N = ctx->nat_elems;
    const dim3 b3(32, 4, 2), g3 = grid3(g, b3);
    const dim3 b3s(32, 2, 2), g3s = grid3(g, b3s);   // 128-thread blocks
    CK(cudaMemsetAsync(A.lpn, 0, N * sizeof(double), st));
    AdjBcArgs ab{};
    ab.lu = A.lu; ab.lv = A.lv; ab.lw = A.lw; ab.lp = A.lp;
    std::memcpy(ab.bc, P.bc, sizeof ab.bc);
    ab.gval = A.gval;
    k_adj_bc_z<<<dim3((g.nx + 4 + 31) / 32, (g.ny + 4 + 7) / 8), dim3(32, 8), 0, st>>>(g, ab);
    k_adj_bc_y<<<dim3((g.nx + 4 + 31) / 32, (g.nz + 4 + 7) / 8), dim3(32, 8), 0, st>>>(g, ab);
    k_adj_bc_x<<<dim3((g.ny + 4 + 31) / 32, (g.nz + 4 + 7) / 8), dim3(32, 8), 0, st>>>(g, ab);
    k_adj_weights<<<g3, b3, 0, st>>>(g, guards, scaleD, scaleL, A.wD, A.wL);
    if (A.geta) {
        // u* of the step again (the forward predictor on the state before it), for u1
        CK(cudaMemcpyAsync(ctx->u, su, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ctx->v, sv, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ctx->w, sw, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        launch_predictor(ctx, st);
        k_adj_eta<<<g3, b3, 0, st>>>(g, A.lu, A.lv, A.lw, A.wD, A.wL, ctx->us, ctx->vs, ctx->ws, pn, po,
                                     P.u_solid[0], P.u_solid[1], P.u_solid[2], P.dt, A.geta);
    }
    k_adj_project1<<<g3, b3, 0, st>>>(g, A.lu, A.lv, A.lw, ctx->eta, A.wD, A.wL, P.dt, A.lus, A.lvs, A.lws);
    k_adj_project2<<<g3, b3, 0, st>>>(g, A.lus, A.lvs, A.lws, P.dt, A.lp, A.lpn);
    k_adj_solve_rhs<<<g3, b3, 0, st>>>(g, ctx->scd, A.lp, A.badj);
    CK(cudaMemsetAsync(A.slot, 0, sizeof(unsigned long long), st));
    k_absmax<256><<<g3, b3, 0, st>>>(g, A.badj, A.slot);
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, A.slot, sizeof bits, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    double bmax;
    std::memcpy(&bmax, &bits, sizeof bmax);
    if (!std::isfinite(bmax)) return fail(ctx, NTCFD_ENONFINITE, "non-finite adjoint pressure right-hand side");
    if (bmax > 0.0) {
        if (A.solves >= 2) k_extrapolate<<<g3, b3, 0, st>>>(g, A.z, A.zprev);
        else CK(cudaMemcpyAsync(A.zprev, A.z, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        Ctl h{};
        CK(cudaEventRecord(A.e0, st));
        if (int rc = sor_solve_eager<Tc>(ctx, A.z, A.badj, zeta_rel * bmax, itmax, omega, &h, kAdjQueued))
            return rc;
        CK(cudaEventRecord(A.e1, st));
        CK(cudaEventSynchronize(A.e1));
        float sms = 0.0f;
        CK(cudaEventElapsedTime(&sms, A.e0, A.e1));
        A.solve_ms += sms;
        A.solves += 1;
        if (h.timeout) return fail(ctx, NTCFD_ETIMEOUT, "the resident SOR kernel's grid barrier gave up waiting");
        if (h.nonfinite) return fail(ctx, NTCFD_ENONFINITE, "non-finite value in an adjoint SOR solve");
        *sweeps += h.ik;
        if (!h.converged) *unconverged += 1;
    } else {
        CK(cudaMemsetAsync(A.z, 0, N * sizeof(double), st));
        CK(cudaMemsetAsync(A.zprev, 0, N * sizeof(double), st));
        A.solves = 0;
    }
    k_adj_after_solve<<<g3, b3, 0, st>>>(g, ctx->scd, A.z, A.lb, A.lpn);
    k_adj_rhs<<<g3, b3, 0, st>>>(g, ctx->scd, A.lb, P.dt, A.lus, A.lvs, A.lws, A.lu, A.lv, A.lw);
    const int aliased = P.smag_mode == NTCFD_SMAG_REF_ALIASED ? 1 : 0;
    if (P.LES) {
        k_smagorinsky<<<g3, b3, 0, st>>>(g, su, sv, sw, ctx->nut, P.Cs, aliased);
        CK(cudaMemsetAsync(A.lnut, 0, N * sizeof(double), st));
    }
    AdjPredArgs pa{su, sv, sw, P.LES ? ctx->nut : nullptr, A.lus, A.lvs, A.lws, A.lu, A.lv, A.lw,
                   P.LES ? A.lnut : nullptr, A.gf, (long long)N, P.dt, 1. / P.Re, P.LES};
    k_adj_predictor<<<g3s, b3s, 0, st>>>(g, ctx->tpd, pa);
    if (P.LES)
        k_adj_smagorinsky<<<g3s, b3s, 0, st>>>(g, su, sv, sw, A.lnut, P.Cs, aliased, A.lu, A.lv, A.lw);
    CK(cudaGetLastError());
    std::swap(A.lp, A.lpn);
    return 0;
}

template <class Tc>
int adjoint_t(ntcfd_ctx* ctx, const ntcfd_adj_spec* sp, ntcfd_adj_result* res, double* gout[3],
              ntcfd_step_info* per_step) {
    const auto t0 = std::chrono::steady_clock::now();
    const Geom g = ctx->g;
    const ntcfd_params& P = ctx->prm;
    cudaStream_t st = ctx->stream;
    const size_t N = ctx->nat_elems;
    const int K = sp->nsteps, M = sp->checkpoint_every;
    const int nck = (K + M - 1) / M;
    const size_t G = 2 * (size_t)g.nx * g.ny + 2 * (size_t)g.nx;   // guard bytes per step
    const size_t fyz = (size_t)g.ny * g.nz, fxz = (size_t)g.nx * g.nz, fxy = (size_t)g.nx * g.ny;
    const size_t nface = 2 * (fyz + fxz + fxy);
    struct Events {
        cudaEvent_t a = nullptr, b = nullptr, c = nullptr, d = nullptr;
        ~Events() {
            for (cudaEvent_t e : {a, b, c, d})
                if (e) cudaEventDestroy(e);
        }
    } ev;
    CK(cudaEventCreate(&ev.a));
    CK(cudaEventCreate(&ev.b));
    CK(cudaEventCreate(&ev.c));
    CK(cudaEventCreate(&ev.d));
    double *ckpt, *blk, *fin;
    unsigned char* guards;
    AdjBufs A{};
    // with the smoothed mask the steps' pressures are kept too (dJ/dETA needs u1)
    const bool body = ctx->smooth_active;
    const size_t bw = body ? 4 : 3;
    A.e0 = ev.a;
    A.e1 = ev.b;
    double** lam[] = {&A.lu, &A.lv, &A.lw, &A.lp, &A.lpn, &A.lus, &A.lvs, &A.lws, &A.z, &A.zprev, &A.badj,
                      &A.lb, &A.wD, &A.wL};
    auto carve = [&](AdjCarve& cv) {
        cv.take(&ckpt, (size_t)nck * 4 * N);
        cv.take(&blk, (size_t)M * bw * N);
        cv.take(&fin, 4 * N + nface);
        cv.take(&guards, (size_t)K * G);
        for (double** q : lam) cv.take(q, N);
        cv.take(&A.lnut, P.LES ? N : 1);
        cv.take(&A.gf, 3 * N);
        cv.take(&A.gval, 18);
        cv.take(&A.slot, 1);
        cv.take(&A.geta, body ? N : 1);
        cv.take(&A.etacol, body ? (size_t)g.ny * g.nz : 1);
    };
    {
        AdjCarve sizing;
        carve(sizing);
        if (sizing.off > ctx->adj_cap) {
            if (ctx->adj_buf) {
                CK(cudaStreamSynchronize(st));
                cudaFree(ctx->adj_buf);
                ctx->adj_buf = nullptr;
                ctx->adj_cap = 0;
            }
            CK(cudaMalloc(&ctx->adj_buf, sizing.off));
            ctx->adj_cap = sizing.off;
        }
        AdjCarve real;
        real.base = static_cast<char*>(ctx->adj_buf);
        carve(real);
    }
    for (double** q : lam) CK(cudaMemsetAsync(*q, 0, N * sizeof(double), st));
    CK(cudaMemsetAsync(A.gf, 0, 3 * N * sizeof(double), st));
    if (body) CK(cudaMemsetAsync(A.geta, 0, N * sizeof(double), st));
    else A.geta = nullptr;
    CK(cudaMemsetAsync(A.gval, 0, 18 * sizeof(double), st));
    if (int rc = prepare_steps(ctx, std::max(K, M))) return rc;
    auto save_state = [&](double* dst) -> int {
        double* src[4] = {ctx->u, ctx->v, ctx->w, ctx->p};
        for (int q = 0; q < 4; ++q)
            CK(cudaMemcpyAsync(dst + q * N, src[q], N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        return 0;
    };
    auto load_state = [&](const double* srcb) -> int {
        double* dst[4] = {ctx->u, ctx->v, ctx->w, ctx->p};
        for (int q = 0; q < 4; ++q)
            CK(cudaMemcpyAsync(dst[q], srcb + q * N, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        return 0;
    };
    double* faces[6] = {ctx->faceW, ctx->faceE, ctx->faceS, ctx->faceN, ctx->faceB, ctx->faceF};
    const size_t flen[6] = {fyz, fyz, fxz, fxz, fxy, fxy};
    BcArgs ba{};
    ba.u = ctx->u; ba.v = ctx->v; ba.w = ctx->w; ba.p = ctx->p;
    std::memcpy(ba.bc, P.bc, sizeof ba.bc);
    std::memcpy(ba.val, P.bc_value, sizeof ba.val);
    ba.faceW = ctx->faceW; ba.faceE = ctx->faceE; ba.faceS = ctx->faceS;
    ba.faceN = ctx->faceN; ba.faceB = ctx->faceB; ba.faceF = ctx->faceF;
    const dim3 gbx((g.ny + 4 + 31) / 32, (g.nz + 4 + 7) / 8), gby((g.nx + 4 + 31) / 32, (g.nz + 4 + 7) / 8),
        gbz((g.nx + 4 + 31) / 32, (g.ny + 4 + 7) / 8), bbc(32, 8);
    if (sp->initial_bc) {
        k_bc_x<<<bc_grid_x(g), bbc, 0, st>>>(g, ba);
        k_bc_y<<<bc_grid_y(g), bbc, 0, st>>>(g, ba);
        k_bc_z<<<bc_grid_z(g), bbc, 0, st>>>(g, ba);
        CK(cudaGetLastError());
    }
    // ---- forward pass: K steps, a checkpoint every M, the guards of every step
    CK(cudaMemsetAsync(&ctx->ctl->step, 0, sizeof(int), st));
    CK(cudaEventRecord(ctx->ev0, st));
    const int last0 = (nck - 1) * M;   // first step of the last block: its states are kept here
    for (int s = 0; s < K; ++s) {
        if (s % M == 0)
            if (int rc = save_state(ckpt + (size_t)(s / M) * 4 * N)) return rc;
        if (s >= last0) {
            double* dst = blk + (size_t)(s - last0) * bw * N;
            CK(cudaMemcpyAsync(dst, ctx->u, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(dst + N, ctx->v, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(dst + 2 * N, ctx->w, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            if (body) CK(cudaMemcpyAsync(dst + 3 * N, ctx->p, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        if (int rc = launch_step(ctx)) return rc;
        k_pack_guards<<<148, 256, 0, st>>>(g, ctx->FXz, ctx->FYz, ctx->FXy, ctx->FYy, guards + (size_t)s * G);
    }
    CK(cudaEventRecord(ctx->ev1, st));
    CK(cudaGetLastError());
    std::vector<StepRec> rec(K);
    CK(cudaMemcpyAsync(rec.data(), ctx->rec, sizeof(StepRec) * K, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float fms = 0.0f;
    CK(cudaEventElapsedTime(&fms, ctx->ev0, ctx->ev1));
    res->forward_ms = fms;
    const int fst = records_to_info(ctx, rec.data(), K, per_step);
    if (fst < 0) return fst;
    res->fwd_status = fst;
    double J = 0.0;
    for (int s = 0; s < K; ++s) J += sp->w_drag * rec[s].cdrag + sp->w_lift * rec[s].clift;
    res->J = J / K;
    if (int rc = save_state(fin)) return rc;
    {
        size_t off = 4 * N;
        for (int q = 0; q < 6; ++q) {
            CK(cudaMemcpyAsync(fin + off, faces[q], flen[q] * sizeof(double), cudaMemcpyDeviceToDevice, st));
            off += flen[q];
        }
    }
    // ---- reverse pass, block by block from the last checkpoint
    const double scaleD = sp->w_drag * (-2.0 / P.lx) / K;
    const double scaleL = sp->w_lift * (-2.0 / P.lx) / K;
    const double zrel = sp->adj_zeta > 0 ? sp->adj_zeta : 1e-7;
    const int itmax = sp->adj_itmax > 0 ? sp->adj_itmax : 20000;
    const double omega = sp->adj_omega > 0 ? sp->adj_omega : 1.9;
    long long sweeps = 0;
    int unconv = 0, recomputed = 0;
    double rms = 0.0;
    for (int b = nck - 1; b >= 0; --b) {
        const int s0 = b * M, s1 = std::min(K, s0 + M);
        if (int rc = load_state(ckpt + (size_t)b * 4 * N)) return rc;
        CK(cudaMemsetAsync(&ctx->ctl->step, 0, sizeof(int), st));
        CK(cudaEventRecord(ev.c, st));
        for (int m = 0; m < s1 - s0 && b < nck - 1; ++m) {
            double* dst = blk + (size_t)m * bw * N;
            CK(cudaMemcpyAsync(dst, ctx->u, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(dst + N, ctx->v, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            CK(cudaMemcpyAsync(dst + 2 * N, ctx->w, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            if (body) CK(cudaMemcpyAsync(dst + 3 * N, ctx->p, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
            if (m + 1 < s1 - s0) {
                if (int rc = launch_step(ctx)) return rc;
                ++recomputed;
            }
        }
        CK(cudaEventRecord(ev.d, st));
        CK(cudaEventSynchronize(ev.d));
        float bms = 0.0f;
        CK(cudaEventElapsedTime(&bms, ev.c, ev.d));
        rms += bms;
        for (int n = s1 - 1; n >= s0; --n) {
            const double* sb = blk + (size_t)(n - s0) * bw * N;
            // the pressure after step n: before step n+1 (this block, the next checkpoint, or the end)
            const double* pn = !body ? nullptr
                               : n + 1 < s1 ? blk + (size_t)(n + 1 - s0) * bw * N + 3 * N
                               : n + 1 < K  ? ckpt + (size_t)(b + 1) * 4 * N + 3 * N
                                            : fin + 3 * N;
            if (int rc = adjoint_step<Tc>(ctx, A, sb, sb + N, sb + 2 * N, body ? sb + 3 * N : nullptr, pn,
                                          guards + (size_t)n * G, scaleD, scaleL, zrel, itmax, omega, &sweeps,
                                          &unconv))
                return rc;
        }
    }
    if (sp->initial_bc) {
        // the initial boundary conditions, transposed (lam of the state before them is not kept)
        AdjBcArgs ab{};
        ab.lu = A.lu; ab.lv = A.lv; ab.lw = A.lw; ab.lp = A.lp;
        std::memcpy(ab.bc, P.bc, sizeof ab.bc);
        ab.gval = A.gval;
        k_adj_bc_z<<<gbz, bbc, 0, st>>>(g, ab);
        k_adj_bc_y<<<gby, bbc, 0, st>>>(g, ab);
        k_adj_bc_x<<<gbx, bbc, 0, st>>>(g, ab);
        CK(cudaGetLastError());
    }
    // ---- results
    double gv[18];
    CK(cudaMemcpyAsync(gv, A.gval, sizeof gv, cudaMemcpyDeviceToHost, st));
    const size_t n = (size_t)g.nx * g.ny * g.nz;
    const dim3 b3(32, 4, 2);
    for (int c = 0; c < 3; ++c) {
        if (!gout[c]) continue;
        k_interior_out<<<grid3(g, b3), b3, 0, st>>>(g, A.gf + c * N, ctx->outbuf);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(gout[c], ctx->outbuf, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    // dJ/dAOA through the body: sum over the cells of dJ/dETA dETA/dAOA
    res->dJ_daoa_body = 0.0;
    if (body) {
        const size_t cells = (size_t)g.ny * g.nz;
        k_colsum_i<<<dim3((g.nz + 31) / 32, (g.ny + 7) / 8), dim3(32, 8), 0, st>>>(g, A.geta, A.etacol);
        CK(cudaGetLastError());
        std::vector<double> col(cells), de(cells);
        CK(cudaMemcpyAsync(col.data(), A.etacol, cells * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(de.data(), ctx->deta_daoa, cells * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double sum = 0.0;
        for (size_t q = 0; q < cells; ++q) sum += col[q] * de[q];
        res->dJ_daoa_body = sum;
    }
    // the state after the K steps, as the forward pass left it
    if (int rc = load_state(fin)) return rc;
    {
        size_t off = 4 * N;
        for (int q = 0; q < 6; ++q) {
            CK(cudaMemcpyAsync(faces[q], fin + off, flen[q] * sizeof(double), cudaMemcpyDeviceToDevice, st));
            off += flen[q];
        }
    }
    CK(cudaStreamSynchronize(st));
    for (int q = 0; q < 18; ++q) res->dJ_dbc[q / 3][q % 3] = gv[q];
    if (sp->inflow_wall >= 0) {
        const double* val = P.bc_value[sp->inflow_wall];
        const double a = val[sp->inflow_normal], t = val[sp->inflow_tangential];
        const double U = std::hypot(a, t), th = std::atan2(t, a);
        const double ga = gv[sp->inflow_wall * 3 + sp->inflow_normal];
        const double gt = gv[sp->inflow_wall * 3 + sp->inflow_tangential];
        res->dJ_dU = ga * std::cos(th) + gt * std::sin(th);
        res->dJ_dtheta = U * (-ga * std::sin(th) + gt * std::cos(th));
    }
    res->recompute_ms = rms;
    res->solve_ms = A.solve_ms;
    res->adj_sweeps = sweeps;
    res->adj_unconverged = unconv;
    res->recomputed_steps = recomputed;
    res->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return unconv ? NTCFD_NOT_CONVERGED : fst;
}

}  // namespace

extern "C" int ntcfd_adjoint(ntcfd_ctx* ctx, const ntcfd_adj_spec* spec, ntcfd_adj_result* result,
                             double* dJ_dfu, double* dJ_dfv, double* dJ_dfw, ntcfd_step_info* per_step) {
    DEV();
    if (!spec || !result) return fail(ctx, NTCFD_EINVAL, "null spec or result");
    std::memset(result, 0, sizeof *result);
    if (!ctx->metrics_set) return fail(ctx, NTCFD_ESTATE, "ntcfd_set_metrics must come before ntcfd_adjoint");
    if (spec->nsteps < 1) return fail(ctx, NTCFD_EINVAL, "nsteps must be >= 1");
    if (ctx->dyn_start > 0)
        return fail(ctx, NTCFD_EINVAL, "the adjoint holds ETA fixed: switch the dynamic angle of attack off");
    if (is_slab(ctx)) return fail(ctx, NTCFD_EINVAL, "the adjoint runs on a single domain, not on a z-slab");
    if (ctx->prm.scheme != NTCFD_QUICK_CENTRE)
        return fail(ctx, NTCFD_EINVAL, "the adjoint differentiates the NTCFD_QUICK_CENTRE predictor only");
    if (spec->checkpoint_every < 1) return fail(ctx, NTCFD_EINVAL, "checkpoint_every must be >= 1");
    if (!(spec->adj_zeta >= 0.0) || spec->adj_itmax < 0) return fail(ctx, NTCFD_EINVAL, "bad adjoint stop rule");
    if (!(spec->adj_omega >= 0.0 && spec->adj_omega < 2.0))
        return fail(ctx, NTCFD_EINVAL, "adj_omega must be in (0, 2), or 0 for the default");
    if (!std::isfinite(spec->w_drag) || !std::isfinite(spec->w_lift))
        return fail(ctx, NTCFD_EINVAL, "non-finite objective weights");
    if (spec->initial_bc != 0 && spec->initial_bc != 1) return fail(ctx, NTCFD_EINVAL, "initial_bc must be 0 or 1");
    for (int r : spec->reserved)
        if (r) return fail(ctx, NTCFD_EINVAL, "reserved fields of ntcfd_adj_spec must be zero");
    if (spec->inflow_wall < -1 || spec->inflow_wall > 5)
        return fail(ctx, NTCFD_EINVAL, "inflow_wall must be -1 or a wall index");
    if (spec->inflow_wall >= 0 &&
        (spec->inflow_normal < 0 || spec->inflow_normal > 2 || spec->inflow_tangential < 0 ||
         spec->inflow_tangential > 2 || spec->inflow_normal == spec->inflow_tangential))
        return fail(ctx, NTCFD_EINVAL, "inflow components must be two distinct indices in 0..2");
    double* gout[3] = {dJ_dfu, dJ_dfv, dJ_dfw};
    const int rc = ctx->prm.precision == NTCFD_MIXED ? adjoint_t<float>(ctx, spec, result, gout, per_step)
                                                     : adjoint_t<double>(ctx, spec, result, gout, per_step);
    if (rc == NTCFD_NOT_CONVERGED && result->adj_unconverged)
        fail(ctx, rc, "%d adjoint pressure solves stopped at adj_itmax", result->adj_unconverged);
    return rc;
}
