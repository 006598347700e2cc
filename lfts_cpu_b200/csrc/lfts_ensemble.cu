// Ensemble of independent FP32-mixed L-FTS replicas advanced together
// (include/lfts_b200.h, "ensemble").  Each replica is an ordinary context
// (buffers, tables, autotuned x-pencil width); the ensemble adds batched
// launches over the replicas of each mesh, the device-side Anderson loop of
// ensemble_kernels.cuh and on-device Philox noise, and captures one whole
// Langevin step of every replica as one CUDA graph:
//
//   [Langevin update, all replicas] -> [begin] -> WHILE (any replica active) {
//       per mesh group, on its own stream: the contour chain in the group's
//       tuned order (enqueue_group_chain)
//       -> Q, concentrations + dots, reduction + least squares, w+ update,
//       control (sets the WHILE condition) }
//
// so a step costs one graph launch and no host round trip.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "ctx.h"
#include "ensemble_kernels.cuh"

using namespace lfts;

extern void lfts_internal_set_error(const char *msg);

namespace {

#define EK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            std::string m_ = std::string(#call) + ": " + cudaGetErrorString(e_);   \
            lfts_internal_set_error(m_.c_str());                                   \
            return LFTS_ERR_CUDA;                                                  \
        }                                                                          \
    } while (0)

using PlaneFn = void (*)(EnsRep *, const int *, int);
using PencilFn = void (*)(EnsRep *, const int *);

struct PlaneSet {
    PlaneFn fn[4];
    int nt;
    size_t smem;
};
struct PencilSet {
    PencilFn fn;
    int nt;
    size_t smem;
};

// meshes (per side) with batched kernels: cubic 16 ... 96
#define LFTS_ENS_LEN(X) X(16) X(24) X(32) X(48) X(64) X(96)

template <int N>
void fill_plane(PlaneSet *o)
{
    using C = PlaneCCfg<float, N, N>;
    o->fn[PLANE_INIT_W] = ens_plane_kernel<N, N, PLANE_INIT_W>;
    o->fn[PLANE_INIT_Q] = ens_plane_kernel<N, N, PLANE_INIT_Q>;
    o->fn[PLANE_STEP] = ens_plane_kernel<N, N, PLANE_STEP>;
    o->fn[PLANE_LAST] = ens_plane_kernel<N, N, PLANE_LAST>;
    o->nt = C::NT;
    o->smem = C::SMEM;
}

template <int N, int CW>
void fill_pencil(PencilSet *o)
{
    using C = PencilCfg<float, N, CW>;
    o->fn = ens_pencil_kernel<N, CW>;
    o->nt = C::NT;
    o->smem = C::SMEM;
}

template <typename C3>
void fill_plane3(PlaneSet *o)
{
    o->fn[PLANE_INIT_W] = ens_plane3_kernel<C3, PLANE_INIT_W>;
    o->fn[PLANE_INIT_Q] = ens_plane3_kernel<C3, PLANE_INIT_Q>;
    o->fn[PLANE_STEP] = ens_plane3_kernel<C3, PLANE_STEP>;
    o->fn[PLANE_LAST] = ens_plane3_kernel<C3, PLANE_LAST>;
    o->nt = C3::NT;
    o->smem = C3::SMEM;
}

// yz-plane kernels of an ensemble mesh: three transform stages per axis
// (fft_plane3.cuh: 64 and 96 planes) or two (fft_packed.cuh), the same bodies
// a single FP32-mixed context runs with those tiles
bool ens_plane(int ny, int nz, int stages, PlaneSet *o)
{
    if (ny != nz) return false;
    if (stages == 3) {
        if (ny == 96) {
            fill_plane3<Plane3_96>(o);
            return true;
        }
        if (ny == 64) {
            fill_plane3<Plane3_64>(o);
            return true;
        }
        return false;
    }
    if (stages != 2) return false;
#define X(n)                    \
    if (ny == n) {              \
        fill_plane<n>(o);       \
        return true;            \
    }
    LFTS_ENS_LEN(X)
#undef X
    return false;
}

// the h-in-pencil chain's x-pencils (96-point lines, as a single context's)
using PencilXFn = void (*)(EnsRep *, const int *, int);
struct PencilXSet {
    PencilXFn fn[kPencilModes];
    PlaneFn plane_g;  // the chain's yz-plane kernel (PLANE_G, three stages)
    int nt;
    size_t smem;
};

template <int N, int CW>
void fill_pencil_x(PencilXSet *o)
{
    using C = PencilCfg<float, N, CW>;
    for (int m = 0; m < kPencilModes; m++) o->fn[m] = nullptr;
    o->fn[PENCIL_INIT_W] = ens_pencil_x_kernel<N, CW, PENCIL_INIT_W>;
    o->fn[PENCIL_H] = ens_pencil_x_kernel<N, CW, PENCIL_H>;
    o->fn[PENCIL_H_LAST] = ens_pencil_x_kernel<N, CW, PENCIL_H_LAST>;
    o->fn[PENCIL_HA] = ens_pencil_x_kernel<N, CW, PENCIL_HA>;
    o->fn[PENCIL_HA_LAST] = ens_pencil_x_kernel<N, CW, PENCIL_HA_LAST>;
    o->plane_g = ens_plane3_kernel<Plane3_96, PLANE_G>;
    o->nt = C::NT;
    o->smem = C::SMEM;
}

// cubic 96^3 replicas only (the plane kernel is the three-stage 96 x 96 one)
bool ens_pencil_x(int nx, int ny, int nz, int cw, PencilXSet *o)
{
    if (nx != 96 || ny != 96 || nz != 96) return false;
    if (cw == 8) { fill_pencil_x<96, 8>(o); return true; }
    if (cw == 16) { fill_pencil_x<96, 16>(o); return true; }
    if (cw == 32) { fill_pencil_x<96, 32>(o); return true; }
    return false;
}

bool ens_pencil(int nx, int cw, PencilSet *o)
{
#define X(n)                                                \
    if (nx == n) {                                          \
        if (cw == 8) { fill_pencil<n, 8>(o); return true; }   \
        if (cw == 16) { fill_pencil<n, 16>(o); return true; } \
        if (cw == 32) { fill_pencil<n, 32>(o); return true; } \
        return false;                                       \
    }
    LFTS_ENS_LEN(X)
#undef X
    return false;
}

struct Group {
    int mx = 0, my = 0, mz = 0, cw = 0, stages = 2;
    int xh = 0, phi = 0;  // h-in-pencil chain; concentration sums in it
    std::vector<int> members;
    int *d_members = nullptr;
    PlaneSet pl{};
    PencilSet pe{};
    PencilXSet px{};
    cudaStream_t st = nullptr;
    cudaEvent_t join = nullptr;
};

}  // namespace

struct lfts_ensemble {
    int dev = 0, nrep = 0, N = 0;
    std::vector<lfts_ctx *> rep;
    std::vector<EnsRep> h_reps;
    EnsRep *d_reps = nullptr;
    std::vector<Group> groups;
    cudaStream_t s0 = nullptr;
    cudaEvent_t fork = nullptr;
    long long *d_step = nullptr;  // Langevin step counter (next step's index)
    double *d_lambda = nullptr;   // 1 - 0.9^k, k < lambda_n
    int lambda_n = 0;
    int max_blocks = 0;           // largest reduction grid of any replica
    // graphs, built for one (maxIter, tol)
    cudaGraph_t g_mix = nullptr, g_run = nullptr;
    cudaGraphExec_t x_mix = nullptr, x_run = nullptr;
    int *d_guard = nullptr;  // body iterations of the current mix (the WHILE node's guard)
    int guard_cap = 0;
    int *d_run = nullptr;    // steps done, steps asked for (the run graph's step loop)
    int *d_kbuf = nullptr;   // Anderson counts of a run, [kbuf_steps][nrep]
    int kbuf_steps = 0;
    int g_maxIter = -1;
    double g_tol = -1.0;
    long long launches = 0;
    std::vector<int> status;  // each replica's status after the last mix / run
};

namespace {

struct EnsDeviceGuard {
    int prev = -1;
    explicit EnsDeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~EnsDeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// one contour chain of every member of group g, on g.st; returns the launches.
// Two chain orders, as a single context's (enqueue_chain_launches):
//   h in the plane: INIT_W plane, N-1 x (x-pencil with g, plane with h storing slot i+1)
//   h in the pencil (96^3): INIT_W pencil, N-1 x (plane with g, pencil with h
//     storing slot i+1 -- or, with the sums in the chain, adding the products
//     with the stored partner slot from the middle on), then Q's plane partials
long long enqueue_group_chain(lfts_ensemble *e, Group &g)
{
    const int nm = (int)g.members.size();
    const dim3 pgrid(g.mx, nm);
    const dim3 egrid((g.my * g.mz + g.cw - 1) / g.cw, nm);
    long long n = 0;
    if (g.xh) {
        g.px.fn[PENCIL_INIT_W]<<<egrid, g.px.nt, g.px.smem, g.st>>>(e->d_reps, g.d_members, 0);
        n++;
        for (int i = 1; i < e->N; i++) {
            g.px.plane_g<<<pgrid, g.pl.nt, g.pl.smem, g.st>>>(e->d_reps, g.d_members, i);
            const int p = e->N - i;  // partner slot
            const bool last = i + 1 == e->N;
            const int mode = (!g.phi || p > i + 1) ? (last ? PENCIL_H_LAST : PENCIL_H)
                                                   : (last ? PENCIL_HA_LAST : PENCIL_HA);
            g.px.fn[mode]<<<egrid, g.px.nt, g.px.smem, g.st>>>(e->d_reps, g.d_members, i);
            n += 2;
        }
        ens_plane_q_sums_kernel<<<pgrid, 256, 0, g.st>>>(e->d_reps, g.d_members);
        return n + 1;
    }
    g.pl.fn[PLANE_INIT_W]<<<pgrid, g.pl.nt, g.pl.smem, g.st>>>(e->d_reps, g.d_members, 0);
    n++;
    for (int i = 1; i < e->N; i++) {
        g.pe.fn<<<egrid, g.pe.nt, g.pe.smem, g.st>>>(e->d_reps, g.d_members);
        g.pl.fn[i + 1 < e->N ? PLANE_STEP : PLANE_LAST]<<<pgrid, g.pl.nt, g.pl.smem, g.st>>>(e->d_reps, g.d_members,
                                                                                           i);
        n += 2;
    }
    return n;
}

// one iteration of every active replica, enqueued on e->s0 (being captured)
int enqueue_body(lfts_ensemble *e, int maxIter, double tol, cudaGraphConditionalHandle loop)
{
    EK(cudaEventRecord(e->fork, e->s0));
    for (Group &g : e->groups) {
        EK(cudaStreamWaitEvent(g.st, e->fork, 0));
        e->launches += enqueue_group_chain(e, g);
        EK(cudaGetLastError());
        EK(cudaEventRecord(g.join, g.st));
        EK(cudaStreamWaitEvent(e->s0, g.join, 0));
    }
    ens_qfinal_kernel<<<e->nrep, 256, 0, e->s0>>>(e->d_reps);
    ens_conc_kernel<<<dim3(e->max_blocks, e->nrep), kRedThreads, 0, e->s0>>>(e->d_reps, nullptr);
    ens_reduce_solve_kernel<<<e->nrep, 256, 0, e->s0>>>(e->d_reps, tol, maxIter);
    ens_update_kernel<<<dim3(e->max_blocks, e->nrep), 256, 0, e->s0>>>(e->d_reps, e->d_lambda);
    ens_control_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep, loop, e->d_guard, e->guard_cap);
    e->launches += 5;
    EK(cudaGetLastError());
    return LFTS_OK;
}

// A WHILE node running enqueue_body (the Anderson loop of every replica),
// added to graph g after node `dep` (null: no dependency); *loop_out is its
// handle, created in g.
int add_mix_loop(lfts_ensemble *e, cudaGraph_t g, cudaGraphNode_t dep, int maxIter, double tol,
                 cudaGraphConditionalHandle loop, cudaGraphNode_t *node_out)
{
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    EK(cudaGraphAddNode(node_out, g, &dep, dep ? 1 : 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    EK(cudaStreamBeginCaptureToGraph(e->s0, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_body(e, maxIter, tol, loop);
    cudaGraph_t body_out = nullptr;
    cudaError_t ce = cudaStreamEndCapture(e->s0, &body_out);
    if (rc) return rc;
    EK(ce);
    return LFTS_OK;
}

// the node of g without dependents (the end of a captured prologue)
int last_node(cudaGraph_t g, cudaGraphNode_t *out)
{
    size_t nn = 0;
    EK(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    EK(cudaGraphGetNodes(g, nodes.data(), &nn));
    *out = nullptr;
    for (cudaGraphNode_t n : nodes) {
        size_t nd = 0;
        EK(cudaGraphNodeGetDependentNodes(n, nullptr, &nd));
        if (nd == 0) *out = n;
    }
    return LFTS_OK;
}

int finish_graph(lfts_ensemble *e, cudaGraph_t g, cudaGraphExec_t *x_out)
{
    cudaGraphExec_t x = nullptr;
    EK(cudaGraphInstantiate(&x, g, 0));
    EK(cudaGraphUpload(x, e->s0));
    EK(cudaStreamSynchronize(e->s0));
    *x_out = x;
    return LFTS_OK;
}

void langevin_launch(lfts_ensemble *e)
{
    long long maxM = 0;
    for (const EnsRep &r : e->h_reps) maxM = std::max(maxM, r.M);
    const int lb = (int)std::min<long long>((maxM + 255) / 256, 1184);
    ens_langevin_kernel<<<dim3(lb, e->nrep), 256, 0, e->s0>>>(e->d_reps, e->d_step);
}

// the mix graph: begin -> WHILE(body)
int build_mix_graph(lfts_ensemble *e, int maxIter, double tol, cudaGraph_t *g_out, cudaGraphExec_t *x_out)
{
    cudaGraph_t g = nullptr;
    EK(cudaGraphCreate(&g, 0));
    auto fail = [&](int rc) {
        cudaGraphDestroy(g);
        return rc;
    };
    cudaGraphConditionalHandle loop;
    if (cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    if (cudaStreamBeginCaptureToGraph(e->s0, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    ens_begin_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep, e->d_step, 0, e->d_guard, 0, 0);
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(e->s0, &captured) != cudaSuccess) return fail(LFTS_ERR_CUDA);
    cudaGraphNode_t last = nullptr, cond = nullptr;
    int rc = last_node(g, &last);
    if (!rc) rc = add_mix_loop(e, g, last, maxIter, tol, loop, &cond);
    if (!rc) rc = finish_graph(e, g, x_out);
    if (rc) return fail(rc);
    *g_out = g;
    return LFTS_OK;
}

// the run graph, one launch for a whole run of Langevin steps:
//   WHILE (steps done < steps asked) {
//       Langevin update -> begin (raises the mix condition) -> WHILE(mix body) -> step end
//   }
// the step loop's handle belongs to the top graph, the mix loop's to the
// step loop's body
int build_run_graph(lfts_ensemble *e, int maxIter, double tol, cudaGraph_t *g_out, cudaGraphExec_t *x_out)
{
    cudaGraph_t g = nullptr;
    EK(cudaGraphCreate(&g, 0));
    auto fail = [&](int rc) {
        cudaGraphDestroy(g);
        return rc;
    };
    cudaGraphConditionalHandle outer;
    if (cudaGraphConditionalHandleCreate(&outer, g, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = outer;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t outer_node = nullptr;
    if (cudaGraphAddNode(&outer_node, g, nullptr, 0, &cp) != cudaSuccess) return fail(LFTS_ERR_CUDA);
    cudaGraph_t steps = cp.conditional.phGraph_out[0];
    cudaGraphConditionalHandle inner;
    if (cudaGraphConditionalHandleCreate(&inner, steps, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    // step prologue: Langevin update of every replica, begin of the mix
    if (cudaStreamBeginCaptureToGraph(e->s0, steps, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    langevin_launch(e);
    ens_begin_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep, e->d_step, 1, e->d_guard, 1, inner);
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(e->s0, &captured) != cudaSuccess) return fail(LFTS_ERR_CUDA);
    cudaGraphNode_t last = nullptr, mix = nullptr;
    int rc = last_node(steps, &last);
    if (!rc) rc = add_mix_loop(e, steps, last, maxIter, tol, inner, &mix);
    if (rc) return fail(rc);
    // step end, after the mix loop
    if (cudaStreamBeginCaptureToGraph(e->s0, steps, &mix, nullptr, 1, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    ens_step_end_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep, e->d_run, e->d_kbuf, outer);
    if (cudaStreamEndCapture(e->s0, &captured) != cudaSuccess) return fail(LFTS_ERR_CUDA);
    if ((rc = finish_graph(e, g, x_out))) return fail(rc);
    *g_out = g;
    return LFTS_OK;
}

void drop_graphs(lfts_ensemble *e)
{
    if (e->x_mix) cudaGraphExecDestroy(e->x_mix);
    if (e->x_run) cudaGraphExecDestroy(e->x_run);
    if (e->g_mix) cudaGraphDestroy(e->g_mix);
    if (e->g_run) cudaGraphDestroy(e->g_run);
    e->x_mix = e->x_run = nullptr;
    e->g_mix = e->g_run = nullptr;
}

int ensure_graphs(lfts_ensemble *e, int maxIter, double tol)
{
    if (e->x_mix && e->g_maxIter == maxIter && e->g_tol == tol) return LFTS_OK;
    drop_graphs(e);
    // lambda_k = 1 - 0.9^k (src/anderson.cc:44), host pow as in the single context
    std::vector<double> lam(maxIter + 2);
    for (int k = 0; k < (int)lam.size(); k++) lam[k] = 1.0 - std::pow(0.9, double(k));
    if (e->d_lambda) cudaFree(e->d_lambda);
    e->d_lambda = nullptr;
    EK(cudaMalloc(&e->d_lambda, sizeof(double) * lam.size()));
    EK(cudaMemcpy(e->d_lambda, lam.data(), sizeof(double) * lam.size(), cudaMemcpyHostToDevice));
    e->lambda_n = (int)lam.size();
    e->guard_cap = maxIter + 2;
    int rc = build_mix_graph(e, maxIter, tol, &e->g_mix, &e->x_mix);
    if (!rc) rc = build_run_graph(e, maxIter, tol, &e->g_run, &e->x_run);
    if (rc) {
        drop_graphs(e);
        return rc;
    }
    e->g_maxIter = maxIter;
    e->g_tol = tol;
    return LFTS_OK;
}

// ---- batched tile choice ---------------------------------------------------------
// Each mesh group's tiles (x-pencil width 8/16/32; yz-plane stages 3 or 2 where
// both exist; at 96^3 also the h-in-pencil chain, with or without the
// concentration sums in it) are picked by timing the group's batched contour
// chain and concentration pass, all its replicas active, on its own stream --
// batched, the best tiles differ from a single context's (the plane launches
// run in several waves) -- once per (mesh, group size, N) per process.  The
// choice is installed in every member context too, so lfts_get_tiles on a
// replica's context, or lfts_set_tiles on a single context, gives exactly the
// tiles the replica computes with.
struct GroupTiles {
    int cw, stages, xh, phi;
};
std::mutex g_ens_tune_mu;
std::map<std::tuple<int, int, int, int, int>, GroupTiles> g_ens_tuned;

int set_group_tiles(Group &g, const GroupTiles &t)
{
    PlaneSet pl{};
    PencilSet pe{};
    PencilXSet px{};
    if (!ens_plane(g.my, g.mz, t.stages, &pl) || !ens_pencil(g.mx, t.cw, &pe)) return LFTS_ERR_UNSUPPORTED;
    if (t.phi && !t.xh) return LFTS_ERR_UNSUPPORTED;
    if (t.xh && (t.stages != 3 || !ens_pencil_x(g.mx, g.my, g.mz, t.cw, &px))) return LFTS_ERR_UNSUPPORTED;
    for (int m = 0; m < 4; m++)
        EK(cudaFuncSetAttribute(pl.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem));
    EK(cudaFuncSetAttribute(pe.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pe.smem));
    if (t.xh) {
        EK(cudaFuncSetAttribute(px.plane_g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem));
        for (int m = 0; m < kPencilModes; m++)
            if (px.fn[m])
                EK(cudaFuncSetAttribute(px.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)px.smem));
    }
    g.pl = pl;
    g.pe = pe;
    g.px = px;
    g.cw = t.cw;
    g.stages = t.stages;
    g.xh = t.xh;
    g.phi = t.phi;
    return LFTS_OK;
}

// the group's tiles into its member contexts, and each member's sum buffer
// (allocated by the context when its tiles form the sums in the chain) into
// its device descriptor
int install_group_tiles(lfts_ensemble *e, const Group &g)
{
    const lfts_tiles t{g.cw, g.stages, g.xh, 0, g.phi, 1};
    for (int r : g.members) {
        int rc = lfts_set_tiles(e->rep[r], &t);
        if (rc) return rc;
        float *acc = g.phi ? static_cast<float *>(e->rep[r]->acc) : nullptr;
        if (g.phi && !acc) return LFTS_ERR_NOMEM;
        e->h_reps[r].acc = acc;
        EK(cudaMemcpy(reinterpret_cast<char *>(e->d_reps + r) + offsetof(EnsRep, acc), &acc, sizeof(acc),
                      cudaMemcpyHostToDevice));
    }
    return LFTS_OK;
}

std::vector<GroupTiles> group_candidates(const Group &g)
{
    const char *fcw = std::getenv("LFTS_PENCIL_CW");
    const char *fxh = std::getenv("LFTS_XH_CHAIN");
    const char *fphi = std::getenv("LFTS_PHI_IN_CHAIN");
    const int cw_forced = fcw ? std::atoi(fcw) : 0;
    std::vector<GroupTiles> out;
    PencilXSet px{};
    for (int stages : {3, 2})
        for (int cw : {8, 16, 32}) {
            if (cw_forced > 0 && cw != cw_forced) continue;
            for (int xh : {0, 1}) {
                if (xh && (stages != 3 || !ens_pencil_x(g.mx, g.my, g.mz, cw, &px))) continue;
                if (fxh && ((fxh[0] != '0') != (xh == 1))) continue;
                for (int phi : {0, 1}) {
                    if (phi && !xh) continue;
                    if (fphi && xh && ((fphi[0] != '0') != (phi == 1))) continue;
                    out.push_back({cw, stages, xh, phi});
                }
            }
        }
    return out;
}

int tune_groups(lfts_ensemble *e)
{
    const char *off = std::getenv("LFTS_AUTOTUNE");
    // every replica active, so that the batched kernels do their work
    ens_begin_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep, e->d_step, 0, nullptr, 0, 0);
    EK(cudaStreamSynchronize(e->s0));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    EK(cudaEventCreate(&e0));
    EK(cudaEventCreate(&e1));
    int rc = LFTS_OK;
    for (Group &g : e->groups) {
        const auto key = std::make_tuple(g.mx, g.my, g.mz, (int)g.members.size(), e->N);
        const std::vector<GroupTiles> cand = group_candidates(g);
        if (cand.empty()) {
            rc = LFTS_ERR_UNSUPPORTED;
            break;
        }
        // without timing: 16 columns (or the forced width), three stages where
        // they exist, h in the plane
        const char *fcw = std::getenv("LFTS_PENCIL_CW");
        const int cw_def = fcw && std::atoi(fcw) > 0 ? std::atoi(fcw) : 16;
        GroupTiles best = cand.front();
        for (const GroupTiles &t : cand)
            if (t.cw == cw_def && !t.xh) {
                best = t;
                break;
            }
        if (!(off && off[0] == '0')) {
            std::lock_guard<std::mutex> lk(g_ens_tune_mu);
            auto it = g_ens_tuned.find(key);
            if (it != g_ens_tuned.end()) {
                best = it->second;
            } else {
                float best_ms = 0.f;
                bool found = false;
                const dim3 cgrid(e->max_blocks, (unsigned)g.members.size());
                for (const GroupTiles &t : cand) {
                    if (set_group_tiles(g, t) != LFTS_OK) continue;
                    if ((rc = install_group_tiles(e, g))) break;
                    auto once = [&] {
                        enqueue_group_chain(e, g);
                        ens_conc_kernel<<<cgrid, kRedThreads, 0, g.st>>>(e->d_reps, g.d_members);
                    };
                    once();  // warm-up
                    cudaEventRecord(e0, g.st);
                    for (int r = 0; r < 3; r++) once();
                    cudaEventRecord(e1, g.st);
                    cudaError_t ce = cudaEventSynchronize(e1);
                    if (ce == cudaSuccess) ce = cudaGetLastError();
                    float ms = 0.f;
                    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
                    if (ce != cudaSuccess) {
                        lfts_internal_set_error(cudaGetErrorString(ce));
                        rc = LFTS_ERR_CUDA;
                        break;
                    }
                    if (const char *v = std::getenv("LFTS_VERBOSE"))
                        if (v[0] == '1')
                            fprintf(stderr, "lfts: ensemble group %dx%dx%d (%d replicas) cw %d stages %d h_in_pencil %d "
                                    "phi_in_chain %d: %.4f ms per chain + concentrations\n",
                                    g.mx, g.my, g.mz, (int)g.members.size(), t.cw, t.stages, t.xh, t.phi, ms / 3.0f);
                    if (!found || ms < best_ms) {
                        best_ms = ms;
                        best = t;
                        found = true;
                    }
                }
                if (rc) break;
                if (found) g_ens_tuned[key] = best;
            }
        }
        if ((rc = set_group_tiles(g, best))) break;
        if ((rc = install_group_tiles(e, g))) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

int read_back(lfts_ensemble *e, int *k_out, double *lnQ_out)
{
    EK(cudaStreamSynchronize(e->s0));
    EK(cudaMemcpy(e->h_reps.data(), e->d_reps, sizeof(EnsRep) * e->nrep, cudaMemcpyDeviceToHost));
    // the most severe replica status: non-finite residual, singular system,
    // iteration cap (each replica's own status: lfts_ensemble_replica_status)
    int worst = LFTS_OK, worst_r = -1;
    auto rank = [](int s) { return s == LFTS_ERR_NONFINITE ? 3 : s == LFTS_ERR_SINGULAR ? 2 : s ? 1 : 0; };
    for (int r = 0; r < e->nrep; r++) {
        const EnsRep &R = e->h_reps[r];
        if (k_out) k_out[r] = R.iters;
        const int s = (R.sticky & 4) ? LFTS_ERR_NONFINITE : (R.sticky & 2) ? LFTS_ERR_SINGULAR
                                                          : (R.sticky & 9) ? LFTS_ERR_NOTCONV : LFTS_OK;
        e->status[r] = s;
        if (rank(s) > rank(worst)) {
            worst = s;
            worst_r = r;
        }
        if (lnQ_out) EK(cudaMemcpy(&lnQ_out[r], R.Qd + 1, sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (worst != LFTS_OK) {
        const char *what = worst == LFTS_ERR_NONFINITE ? "a NaN or infinite Anderson residual"
                           : worst == LFTS_ERR_SINGULAR ? "a singular Anderson least-squares matrix"
                                                        : "Anderson mixing stopped at maxIter above the tolerance";
        lfts_internal_set_error((std::string(what) + " in replica " + std::to_string(worst_r)).c_str());
    }
    return worst;
}

}  // namespace

extern "C" {

int lfts_ensemble_create(const lfts_params *params, const unsigned long long *seeds, int nrep, int device,
                         lfts_ensemble **out)
{
    if (!params || !seeds || nrep < 1 || !out) return LFTS_ERR_ARG;
    *out = nullptr;
    for (int r = 0; r < nrep; r++) {
        const lfts_params &p = params[r];
        if (p.N != params[0].N) {
            lfts_internal_set_error("ensemble replicas must share the chain length N");
            return LFTS_ERR_ARG;
        }
        PlaneSet ps;
        PencilSet qs;
        if (!ens_plane(p.m[1], p.m[2], 2, &ps) || !ens_pencil(p.m[0], 16, &qs)) {
            lfts_internal_set_error("ensemble meshes: 16, 24, 32, 48, 64 or 96 points per side, cubic planes");
            return LFTS_ERR_UNSUPPORTED;
        }
    }
    EnsDeviceGuard dg(device);
    lfts_ensemble *e = new lfts_ensemble();
    e->dev = device;
    e->nrep = nrep;
    e->N = params[0].N;
    auto fail = [&](int code) {
        lfts_ensemble_destroy(e);
        return code;
    };
    for (int r = 0; r < nrep; r++) {
        lfts_ctx *c = nullptr;
        int rc = lfts_create(&params[r], LFTS_FP32_MIXED, device, &c);
        if (rc) return fail(rc);
        e->rep.push_back(c);
    }
    e->h_reps.resize(nrep);
    e->status.assign(nrep, LFTS_OK);
    for (int r = 0; r < nrep; r++) {
        lfts_ctx *c = e->rep[r];
        EnsRep &R = e->h_reps[r];
        std::memset(&R, 0, sizeof(R));
        R.mx = c->mx;
        R.my = c->my;
        R.mz = c->mz;
        R.N = c->N;
        R.NA = c->NA;
        R.NB = c->NB;
        R.M = c->M;
        R.red_blocks = c->red_blocks;
        R.XbN = c->p.XbN;
        R.dt = c->p.dt;
        // sigma = sqrt(2 M dt / (C V))  (src/lfts_params.cc:117)
        const double V = c->p.L[0] * c->p.L[1] * c->p.L[2];
        R.sigma = std::sqrt(2.0 * (double)c->M * c->p.dt / (c->p.C * V));
        R.seed = seeds[r];
        R.w = c->w;
        R.q = static_cast<float *>(c->q);
        R.spec = static_cast<cpx<float> *>(c->spec);
        for (int d = 0; d < 3; d++) {
            R.tw[d] = static_cast<const cpx<float> *>(c->tw[d]);
            R.g[d] = static_cast<const float *>(c->gtab[d]);
        }
        R.qpart = c->qpart;
        R.Qd = c->Qd;
        R.partials = c->partials;
        R.acc = nullptr;  // set by the group's tiles (install_group_tiles)
        for (int i = 0; i < kRedWidth; i++) {
            R.Dh[i] = static_cast<float *>(c->Dh[i]);
            R.wh[i] = static_cast<float *>(c->wh[i]);
            R.phys[i] = c->phys[i];
        }
        R.cur = c->cur;
        e->max_blocks = std::max(e->max_blocks, c->red_blocks);
        // group by mesh; the x-pencil width is the context's autotuned one
        int gi = -1;
        for (int g = 0; g < (int)e->groups.size(); g++)
            if (e->groups[g].mx == c->mx && e->groups[g].my == c->my && e->groups[g].mz == c->mz) gi = g;
        if (gi < 0) {
            Group g;
            g.mx = c->mx;
            g.my = c->my;
            g.mz = c->mz;
            g.cw = 16;
            g.stages = 2;
            ens_plane(g.my, g.mz, g.stages, &g.pl);
            if (!ens_pencil(g.mx, g.cw, &g.pe)) return fail(LFTS_ERR_UNSUPPORTED);
            e->groups.push_back(g);
            gi = (int)e->groups.size() - 1;
        }
        e->groups[gi].members.push_back(r);
    }
    if (cudaStreamCreateWithFlags(&e->s0, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(LFTS_ERR_CUDA);
    for (Group &g : e->groups) {
        if (cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&g.d_members, sizeof(int) * g.members.size()) != cudaSuccess ||
            cudaMemcpy(g.d_members, g.members.data(), sizeof(int) * g.members.size(), cudaMemcpyHostToDevice) !=
                cudaSuccess)
            return fail(LFTS_ERR_CUDA);
        for (int m = 0; m < 4; m++)
            if (cudaFuncSetAttribute(g.pl.fn[m], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.pl.smem) !=
                cudaSuccess)
                return fail(LFTS_ERR_CUDA);
        if (cudaFuncSetAttribute(g.pe.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.pe.smem) !=
            cudaSuccess)
            return fail(LFTS_ERR_CUDA);
    }
    const long long step1 = 1;  // step 0 is the initial noise (the langevin constructor's draw)
    if (cudaMalloc(&e->d_reps, sizeof(EnsRep) * nrep) != cudaSuccess ||
        cudaMemcpy(e->d_reps, e->h_reps.data(), sizeof(EnsRep) * nrep, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&e->d_step, sizeof(long long)) != cudaSuccess ||
        cudaMemcpy(e->d_step, &step1, sizeof(long long), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(LFTS_ERR_NOMEM);
    e->kbuf_steps = 1024;
    if (cudaMalloc(&e->d_guard, sizeof(int)) != cudaSuccess || cudaMemset(e->d_guard, 0, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&e->d_run, 2 * sizeof(int)) != cudaSuccess || cudaMemset(e->d_run, 0, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&e->d_kbuf, sizeof(int) * (size_t)e->kbuf_steps * nrep) != cudaSuccess)
        return fail(LFTS_ERR_NOMEM);
    int rc = tune_groups(e);
    if (rc) return fail(rc);
    *out = e;
    return LFTS_OK;
}

int lfts_ensemble_destroy(lfts_ensemble *e)
{
    if (!e) return LFTS_OK;
    EnsDeviceGuard dg(e->dev);
    if (e->s0) cudaStreamSynchronize(e->s0);
    drop_graphs(e);
    for (Group &g : e->groups) {
        if (g.st) cudaStreamDestroy(g.st);
        if (g.join) cudaEventDestroy(g.join);
        cudaFree(g.d_members);
    }
    if (e->s0) cudaStreamDestroy(e->s0);
    if (e->fork) cudaEventDestroy(e->fork);
    cudaFree(e->d_reps);
    cudaFree(e->d_step);
    cudaFree(e->d_lambda);
    cudaFree(e->d_guard);
    cudaFree(e->d_run);
    cudaFree(e->d_kbuf);
    for (lfts_ctx *c : e->rep) lfts_destroy(c);
    delete e;
    return LFTS_OK;
}

int lfts_ensemble_set_fields(lfts_ensemble *e, int r, const double *w_host)
{
    if (!e || r < 0 || r >= e->nrep || !w_host) return LFTS_ERR_ARG;
    EnsDeviceGuard dg(e->dev);
    EK(cudaStreamSynchronize(e->s0));
    return lfts_set_fields(e->rep[r], w_host);
}

int lfts_ensemble_get_fields(lfts_ensemble *e, int r, double *w_host)
{
    if (!e || r < 0 || r >= e->nrep || !w_host) return LFTS_ERR_ARG;
    EnsDeviceGuard dg(e->dev);
    EK(cudaStreamSynchronize(e->s0));
    return lfts_get_fields(e->rep[r], w_host);
}

int lfts_ensemble_mix(lfts_ensemble *e, int maxIter, double tol, int *k_out, double *lnQ_out)
{
    if (!e || maxIter < 2) return LFTS_ERR_ARG;
    EnsDeviceGuard dg(e->dev);
    int rc = ensure_graphs(e, maxIter, tol);
    if (rc) return rc;
    ens_clear_status_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep);
    EK(cudaGraphLaunch(e->x_mix, e->s0));
    return read_back(e, k_out, lnQ_out);
}

int lfts_ensemble_run(lfts_ensemble *e, int nsteps, int maxIter, double tol, int *k_out, double *lnQ_out)
{
    if (!e || nsteps < 0 || maxIter < 2) return LFTS_ERR_ARG;
    EnsDeviceGuard dg(e->dev);
    int rc = ensure_graphs(e, maxIter, tol);
    if (rc) return rc;
    ens_clear_status_kernel<<<1, 256, 0, e->s0>>>(e->d_reps, e->nrep);
    // one graph launch runs up to kbuf_steps steps (the step loop is a WHILE
    // node on the device); the Anderson counts come back once per launch
    for (int s0 = 0; s0 < nsteps; s0 += e->kbuf_steps) {
        const int n = std::min(e->kbuf_steps, nsteps - s0);
        const int run[2] = {0, n};
        EK(cudaMemcpyAsync(e->d_run, run, sizeof(run), cudaMemcpyHostToDevice, e->s0));
        EK(cudaGraphLaunch(e->x_run, e->s0));
        if (k_out)
            EK(cudaMemcpyAsync(k_out + (long long)s0 * e->nrep, e->d_kbuf, sizeof(int) * (size_t)n * e->nrep,
                               cudaMemcpyDeviceToHost, e->s0));
    }
    return read_back(e, nullptr, lnQ_out);
}

int lfts_ensemble_replica_status(const lfts_ensemble *e, int r, int *status)
{
    if (!e || r < 0 || r >= e->nrep || !status) return LFTS_ERR_ARG;
    *status = e->status[r];
    return LFTS_OK;
}

int lfts_ensemble_tuning(const lfts_ensemble *e, int r, int *pencil_cw)
{
    if (!e || r < 0 || r >= e->nrep) return LFTS_ERR_ARG;
    if (pencil_cw) *pencil_cw = e->rep[r]->pe32.cw;
    return LFTS_OK;
}

int lfts_ensemble_tiles(const lfts_ensemble *e, int r, lfts_tiles *out)
{
    if (!e || r < 0 || r >= e->nrep || !out) return LFTS_ERR_ARG;
    return lfts_get_tiles(e->rep[r], out);
}

void *lfts_ensemble_stream(lfts_ensemble *e) { return e ? (void *)e->s0 : nullptr; }

long long lfts_ensemble_kernel_launches(const lfts_ensemble *e) { return e ? e->launches : 0; }

int lfts_noise_philox(unsigned long long seed, long long step, long long n, double sigma, double *out_host)
{
    if (!out_host || n < 0) return LFTS_ERR_ARG;
    if (n == 0) return LFTS_OK;
    double *d = nullptr;
    EK(cudaMalloc(&d, sizeof(double) * n));
    philox_noise_kernel<<<(int)std::min<long long>((n + 255) / 256, 4096), 256>>>(seed, step, n, sigma, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out_host, d, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    EK(e);
    return LFTS_OK;
}

}  // extern "C"
