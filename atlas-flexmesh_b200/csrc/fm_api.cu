// fm_api.cu — the C ABI (include/fm_api.h) over the FlexMesh kernels.
//
// The context owns the mesh structures, the CSR pattern, the stiffness and
// factor buffers and the solver work vectors on one device and stream.
// Host-side loops (PCG iterations, Newton iterations, load steps) launch
// kernels and read back only scalars (norms, stop flags).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "fm_api.h"
#include "fm_devbuf.hpp"
#include "fm_kernels.hpp"
#include "fm_adjoint.hpp"
#include "fm_meshsetup.hpp"
#include "fm_nodes.hpp"
#include "fm_setup.hpp"

namespace {

using fm::DevBuf;

struct SolverCsr {
    uint32_t n = 0;
    uint64_t nnz = 0;
    uint32_t max_row = 0;
    DevBuf<uint32_t> rp, ci, dpos, upos, fwd, bwd;
    std::vector<uint32_t> h_rp, h_ci;
    fm::CsrDev view() const {
        fm::CsrDev v;
        v.n = n;
        v.rp = rp.p;
        v.ci = ci.p;
        v.dpos = dpos.p;
        v.upos = upos.p;
        v.fwd_order = fwd.p;
        v.bwd_order = bwd.p;
        v.max_row = max_row;
        return v;
    }
};

template <typename T>
struct Work {
    DevBuf<T> K, LU, diag, dinv, r, z, p, Ap, t, b, x;
    bool factor_valid = false;
};

}  // namespace

struct fm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    // mesh
    uint32_t nn = 0, ne = 0, n = 0;
    uint64_t nnz = 0;
    std::vector<double> h_xyz;
    std::vector<uint32_t> h_conn;
    std::vector<uint8_t> h_skip;
    fm::NodeGraph graph;
    std::vector<uint32_t> node_lp, node_lo, node_up, node_uo;  // node levels (ptr, order)
    DevBuf<double> xyz;
    DevBuf<uint4> conn;
    DevBuf<uint32_t> nbr_ptr, nbr, inc_ptr, inc_e;
    SolverCsr fem;   // solve pattern of the mesh
    SolverCsr gen;   // generic CSR (fm_csr_pcg_ilu0)
    // node-block schedule of the solve pattern (ILU(0) and triangular solves)
    DevBuf<uint32_t> self_pos, node_fwd, node_bwd, emap_ptr;
    DevBuf<uint8_t> emap;  // ILU(0) update map
    DevBuf<uint4> node_fwd_rec, node_bwd_rec;
    uint32_t node_levels_fwd = 0, node_levels_bwd = 0, width_fwd = 0, width_bwd = 0;
    std::vector<uint32_t> lvl_fwd_ptr, lvl_fwd_rows, lvl_bwd_ptr, lvl_bwd_rows;
    // slab-partitioned push solves (fm_trsv_push.cu): plan on the device and
    // whether they run in FP32 / FP64
    DevBuf<uint32_t> pu_pos_f, pu_pos_b, pu_src, pu_push_f, pu_push_b, pu_nslot_f, pu_nslot_b;
    DevBuf<uint4> pu_rec_f, pu_rec_b;
    fm::PushSolve pu;
    bool pu_ok32 = false, pu_ok64 = false;

    // material
    bool has_mat = false;
    int mat_mode = 0;
    double nu = 0.3, mu_s = 0, lam_s = 0, c_mu = 0, c_lam = 0, inv_cnu = 0;
    DevBuf<double> m0, m1;

    // boundary conditions
    bool has_bc = false, has_bcval = false;
    DevBuf<uint8_t> mask;
    DevBuf<double> bcval;

    // reference-pattern assembly
    DevBuf<int32_t> ref_slot;
    DevBuf<double> ke_scratch;
    DevBuf<unsigned char> elem_rec;  // assembly element-pass records
    DevBuf<uint32_t> inc_pos, nbr_members;  // node-pass scatter structure

    // solver state
    Work<double> w64;
    Work<float> w32;
    DevBuf<double> gen_K, gen_LU, gen_diag;
    DevBuf<unsigned> done;
    unsigned epoch = 0;
    DevBuf<fm::DevScalars> sc;
    fm::DevScalars* h_sc = nullptr;  // pinned mirror
    DevBuf<double> partials;
    DevBuf<double> vec_a, vec_b, vec_c, vec_d, vec_e;  // FP64 scratch (R, du, trial/f, v, host u)
    int grid_trsv64 = 0, grid_trsv32 = 0;

    // built-in profiler: CUDA events around each launch group on the stream
    bool prof_on = false;
    struct ProfRec {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    double prof_ms[FM_PROF_KINDS] = {};
    uint64_t prof_calls[FM_PROF_KINDS] = {};
    uint64_t prof_kernels[FM_PROF_KINDS] = {};

    // per-solve records of the latest Newton call (fm_newton_history)
    std::vector<fm_newton_record> newton_hist;
    // element state arrays updated after every Newton update of u (nullable)
    double* state_F = nullptr;
    double* state_stress = nullptr;

    unsigned* status() { return &sc.p->status; }
    unsigned* counter() { return &sc.p->counter[0]; }
    ~fm_ctx() {
        for (auto& r : prof_pending) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (auto e : prof_pool) cudaEventDestroy(e);
    }
};

namespace {

fm_status fail(fm_ctx* c, fm_status st, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return st;
}

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(c, e_ == cudaErrorMemoryAllocation ? FM_ERR_OOM : FM_ERR_CUDA,     \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define TRY(expr)                       \
    do {                                \
        fm_status s_ = (expr);          \
        if (s_ != FM_OK) return s_;     \
    } while (0)

// ---- profiler ---------------------------------------------------------------
cudaEvent_t prof_event(fm_ctx* c) {
    cudaEvent_t e = nullptr;
    if (!c->prof_pool.empty()) {
        e = c->prof_pool.back();
        c->prof_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        e = nullptr;
    }
    return e;
}
// accumulate completed records (call after the stream was synchronized)
void prof_flush(fm_ctx* c) {
    for (auto& r : c->prof_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) c->prof_ms[r.kind] += ms;
        c->prof_pool.push_back(r.a);
        c->prof_pool.push_back(r.b);
    }
    c->prof_pending.clear();
}
// RAII: records an event pair around the launches of one group of kernels
struct ProfScope {
    fm_ctx* c;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(fm_ctx* ctx, int k, int kernels) : c(ctx), kind(k) {
        c->prof_calls[k] += 1;
        c->prof_kernels[k] += (uint64_t)kernels;
        if (!c->prof_on) return;
        a = prof_event(c);
        if (a) cudaEventRecord(a, c->stream);
    }
    ~ProfScope() {
        if (!a) return;
        cudaEvent_t b = prof_event(c);
        if (!b) {
            c->prof_pool.push_back(a);
            return;
        }
        cudaEventRecord(b, c->stream);
        c->prof_pending.push_back({kind, a, b});
    }
};
#define PROF(kind, nk) ProfScope prof_scope_(c, kind, nk)

template <typename T>
cudaError_t upload(DevBuf<T>& d, const T* h, size_t count, cudaStream_t s) {
    cudaError_t e = d.reserve(count ? count : 1);
    if (e != cudaSuccess) return e;
    if (count) e = cudaMemcpyAsync(d.p, h, count * sizeof(T), cudaMemcpyHostToDevice, s);
    return e;
}

fm_status device_flags(fm_ctx* c, uint32_t* flags) {
    CK(cudaMemcpyAsync(c->h_sc, c->sc.p, sizeof(fm::DevScalars), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->prof_on) prof_flush(c);
    *flags = c->h_sc->status;
    return FM_OK;
}

// The device flags as words, for error texts
std::string flags_text(uint32_t f) {
    static const char* names[] = {"nonfinite", "inverted", "J_clamped", "pivot_perturbed",
                                  "timeout", "breakdown"};
    std::string s;
    for (int b = 0; b < 6; ++b)
        if (f & (1u << b)) {
            if (!s.empty()) s += ",";
            s += names[b];
        }
    return s.empty() ? "none" : s;
}

// Translate fatal device flags into a status
fm_status check_flags(fm_ctx* c, uint32_t flags, const char* where) {
    if (flags & FM_FLAG_TIMEOUT)
        return fail(c, FM_ERR_TIMEOUT, "%s: a bounded dependency wait expired (flags: %s)", where,
                    flags_text(flags).c_str());
    if (flags & FM_FLAG_NONFINITE)
        return fail(c, FM_ERR_NONFINITE, "%s: non-finite value produced (flags: %s)", where,
                    flags_text(flags).c_str());
    return FM_OK;
}

fm_status sync_scalars(fm_ctx* c) {
    CK(cudaMemcpyAsync(c->h_sc, c->sc.p, sizeof(fm::DevScalars), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->prof_on) prof_flush(c);
    return FM_OK;
}

fm::MeshDev mesh_view(const fm_ctx* c) {
    fm::MeshDev m;
    m.n_nodes = c->nn;
    m.n_elems = c->ne;
    m.xyz = c->xyz.p;
    m.conn = c->conn.p;
    m.nbr_ptr = c->nbr_ptr.p;
    m.nbr = c->nbr.p;
    m.inc_ptr = c->inc_ptr.p;
    m.inc = c->inc_e.p;
    m.mask = c->has_bc ? c->mask.p : nullptr;
    m.mat_mode = c->mat_mode;
    m.m0 = c->m0.p;
    m.m1 = c->m1.p;
    m.mu_s = c->mu_s;
    m.lam_s = c->lam_s;
    m.c_mu = c->c_mu;
    m.c_lam = c->c_lam;
    m.inv_cnu = c->inv_cnu;
    m.elem_rec = c->elem_rec.p;
    m.inc_pos = c->inc_pos.p;
    m.nbr_members = c->nbr_members.p;
    return m;
}

// Build the solver CSR (ascending columns) on host and upload: row
// pointers, columns, first-diagonal/first-upper positions and the DOF-level
// dependency orders that the sync-free kernels walk.
fm_status setup_solver_csr(fm_ctx* c, SolverCsr& S, uint32_t n, std::vector<uint32_t>&& rp,
                           std::vector<uint32_t>&& ci) {
    S.n = n;
    S.nnz = rp[n];
    std::vector<uint32_t> dpos(n), upos(n);
    uint32_t max_row = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t k = rp[i];
        while (k < rp[i + 1] && ci[k] < i) ++k;
        dpos[i] = k;
        while (k < rp[i + 1] && ci[k] <= i) ++k;
        upos[i] = k;
        max_row = std::max(max_row, rp[i + 1] - rp[i]);
    }
    S.max_row = max_row;
    std::vector<uint32_t> fp, fr, bp, br;
    fm::csr_levels(n, rp.data(), ci.data(), true, fp, fr);
    fm::csr_levels(n, rp.data(), ci.data(), false, bp, br);
    CK(upload(S.rp, rp.data(), rp.size(), c->stream));
    CK(upload(S.ci, ci.data(), ci.size(), c->stream));
    CK(upload(S.dpos, dpos.data(), n, c->stream));
    CK(upload(S.upos, upos.data(), n, c->stream));
    CK(upload(S.fwd, fr.data(), fr.size(), c->stream));
    CK(upload(S.bwd, br.data(), br.size(), c->stream));
    S.h_rp = std::move(rp);
    S.h_ci = std::move(ci);
    CK(c->done.reserve(std::max<size_t>(c->done.n, n + 1)));
    CK(cudaMemsetAsync(c->done.p, 0, c->done.n * sizeof(unsigned), c->stream));
    c->epoch = 0;
    CK(cudaStreamSynchronize(c->stream));
    return FM_OK;
}

template <typename T>
Work<T>& work(fm_ctx* c);
template <>
Work<double>& work<double>(fm_ctx* c) {
    return c->w64;
}
template <>
Work<float>& work<float>(fm_ctx* c) {
    return c->w32;
}

template <typename T>
fm_status ensure_vectors(fm_ctx* c, uint32_t n) {
    Work<T>& w = work<T>(c);
    CK(w.r.reserve(n));
    CK(w.z.reserve(n));
    CK(w.p.reserve(n));
    CK(w.Ap.reserve(n));
    CK(w.t.reserve(n));
    CK(w.b.reserve(n));
    CK(w.x.reserve(n));
    return FM_OK;
}

unsigned next_epoch(fm_ctx* c) {
    if (++c->epoch == 0) c->epoch = 1;
    return c->epoch;
}

fm::NodeSched node_sched(const fm_ctx* c) {
    fm::NodeSched S;
    S.n_nodes = c->nn;
    S.nbr_ptr = c->nbr_ptr.p;
    S.nbr = c->nbr.p;
    S.self_pos = c->self_pos.p;
    S.fwd_order = c->node_fwd.p;
    S.bwd_order = c->node_bwd.p;
    S.fwd_rec = c->node_fwd_rec.p;
    S.bwd_rec = c->node_bwd_rec.p;
    S.max_width_fwd = c->width_fwd;
    S.max_width_bwd = c->width_bwd;
    S.emap_ptr = c->emap_ptr.p;
    S.emap = c->emap.p;
    return S;
}

// The 16-byte schedule record {node, first neighbour entry, degree, self
// position} of every position of a node order; a hole (~0u) gets node ~0u.
static std::vector<uint4> node_records(const fm::NodeGraph& g, const std::vector<uint32_t>& ord) {
    std::vector<uint4> rec(ord.size());
    for (size_t t = 0; t < ord.size(); ++t) {
        const uint32_t nd = ord[t];
        rec[t] = nd == ~0u ? make_uint4(~0u, 0, 0, 0)
                           : make_uint4(nd, g.ptr[nd], g.ptr[nd + 1] - g.ptr[nd], g.self[nd]);
    }
    return rec;
}

// Plan of the slab-partitioned push solves (fm_trsv_push.cu): one slab per
// thread-block cluster, as many clusters as the device keeps resident (FP32
// and FP64 kernels alike), when every CTA's slots fit its shared memory (the
// plan first tries to fit FP64 slots, else FP32 only) and no node has more
// than 16 neighbours on a side.  The cluster size (8 or 9 CTAs) is the one
// that keeps the most CTAs resident: a cluster must fit in one GPC, and on
// B200 15 clusters of 9 (135 CTAs) are resident against 15 of 8 (measured
// 0.436 against 0.450 ms per FP32 pair, 0.616 against 0.708 FP64, at 64^3).
// The default path; FM_TRSV_PATH=pipe selects the grid-wide pipelined solves
// (fm_trsv.cu) instead.  FM_TRSV_PUSH_WARPS caps the warps per CTA (default:
// 32 in FP32, 16 in FP64), FM_TRSV_PUSH_BLOCK sets the interleave block
// (default: chosen by the plan), FM_TRSV_PUSH_CLUSTER the cluster size.
fm_status setup_push_solves(fm_ctx* c, const std::vector<uint32_t>& lp,
                            const std::vector<uint32_t>& lo, const std::vector<uint32_t>& up,
                            const std::vector<uint32_t>& uo) {
    c->pu_ok32 = c->pu_ok64 = false;
    const char* path = getenv("FM_TRSV_PATH");
    if (path && std::strcmp(path, "push") != 0) return FM_OK;
    // dynamic shared memory per CTA at most; the kernels' static shared
    // memory (under 1 KB) takes the rest of the 227 KB
    constexpr size_t kMaxSmem = 226 * 1024;
    auto env = [](const char* name, int dflt, int lo_, int hi) {
        const char* v = getenv(name);
        return v ? std::min(hi, std::max(lo_, atoi(v))) : dflt;
    };
    const int warps32 = env("FM_TRSV_PUSH_WARPS", fm::push_max_warps(4), 1, fm::push_max_warps(4));
    const int warps64 = std::min(warps32, fm::push_max_warps(8));
    const uint32_t block = (uint32_t)env("FM_TRSV_PUSH_BLOCK", 0, 0, 1 << 20);
    // candidate cluster sizes, most resident CTAs first
    std::vector<std::pair<int, uint32_t>> sizes;  // (resident clusters, size)
    const int forced = env("FM_TRSV_PUSH_CLUSTER", 0, 0, (int)fm::kPushMax);
    for (uint32_t cs = 8; cs <= fm::kPushMax; ++cs) {
        if (forced && cs != (uint32_t)forced) continue;
        const int ncl = std::min(fm::push_max_clusters(4, (int)cs, warps32, kMaxSmem),
                                 fm::push_max_clusters(8, (int)cs, warps64, kMaxSmem));
        if (ncl > 0) sizes.push_back({ncl, cs});
    }
    std::stable_sort(sizes.begin(), sizes.end(), [](const auto& a, const auto& b) {
        return a.first * a.second > b.first * b.second;
    });
    fm::PushPlan p;
    bool planned = false;
    for (const auto& sz : sizes) {
        planned = fm::push_plan(c->graph, lp, lo, up, uo, (uint32_t)sz.first, sz.second, block,
                                (uint32_t)(kMaxSmem / fm::push_smem_bytes(1, 8)), p) ||
                  fm::push_plan(c->graph, lp, lo, up, uo, (uint32_t)sz.first, sz.second, block,
                                (uint32_t)(kMaxSmem / fm::push_smem_bytes(1, 4)), p);
        if (planned) break;
    }
    if (!planned) return FM_OK;
    auto fits = [&](size_t vb) {
        return fm::push_smem_bytes(std::max(p.max_slot_f, p.max_slot_b), vb) <= kMaxSmem;
    };
    const bool ok32 = fits(4), ok64 = fits(8);
    if (!ok32 && !ok64) return FM_OK;
    const std::vector<uint4> rf = node_records(c->graph, p.order_f);
    const std::vector<uint4> rb = node_records(c->graph, p.order_b);
    CK(upload(c->pu_pos_f, p.pos_f.data(), p.pos_f.size(), c->stream));
    CK(upload(c->pu_pos_b, p.pos_b.data(), p.pos_b.size(), c->stream));
    CK(upload(c->pu_src, p.src.data(), p.src.size(), c->stream));
    CK(upload(c->pu_push_f, p.push_f.data(), p.push_f.size(), c->stream));
    CK(upload(c->pu_push_b, p.push_b.data(), p.push_b.size(), c->stream));
    CK(upload(c->pu_nslot_f, p.nslot_f.data(), p.nslot_f.size(), c->stream));
    CK(upload(c->pu_nslot_b, p.nslot_b.data(), p.nslot_b.size(), c->stream));
    CK(upload(c->pu_rec_f, rf.data(), rf.size(), c->stream));
    CK(upload(c->pu_rec_b, rb.data(), rb.size(), c->stream));
    fm::PushSolve v;
    v.n_ctas = p.n_ctas;
    v.cluster = p.cluster;
    v.warps32 = (uint32_t)warps32;
    v.warps64 = (uint32_t)warps64;
    v.max_slot_f = p.max_slot_f;
    v.max_slot_b = p.max_slot_b;
    v.pos_f = c->pu_pos_f.p;
    v.pos_b = c->pu_pos_b.p;
    v.rec_f = c->pu_rec_f.p;
    v.rec_b = c->pu_rec_b.p;
    v.src = c->pu_src.p;
    v.push_f = c->pu_push_f.p;
    v.push_b = c->pu_push_b.p;
    v.nslot_f = c->pu_nslot_f.p;
    v.nslot_b = c->pu_nslot_b.p;

    c->pu = v;
    c->pu_ok32 = ok32;
    c->pu_ok64 = ok64;
    CK(cudaStreamSynchronize(c->stream));
    return FM_OK;
}

// z = U^-1 L^-1 r on the node-block factors (tmp: the intermediate): the
// slab-partitioned push solves where the context has a plan for this value
// width, else the grid-wide pipelined ones.  Returns the kernels launched.
template <typename T>
int precond_nodes(fm_ctx* c, const T* lu, const T* dinv, const T* r, T* tmp, T* z,
                  unsigned* status) {
    const bool pu = sizeof(T) == 4 ? c->pu_ok32 : c->pu_ok64;
    if (pu && c->nn) {
        const cudaError_t e =
            fm::launch_trsv_push<T>(c->pu, node_sched(c), lu, dinv, r, tmp, z, status, c->stream);
        if (e == cudaSuccess) return z != r ? 3 : 4;
        // a launch the device refuses: the pipelined solves from now on
        cudaGetLastError();
        c->pu_ok32 = c->pu_ok64 = false;
    }
    fm::launch_trsv_nodes<T>(node_sched(c), lu, dinv, r, tmp, z, status, c->device, c->stream);
    return 4;
}

// A linear operator for PCG: the mesh K (node-block SpMV) or a generic CSR.
template <typename T>
struct Op {
    fm_ctx* c;
    SolverCsr* S;
    bool node_block;
    const T* K;
    const T* LU;
    const T* diag;
    T* tmp;
    int grid_trsv;
    const T* dinv = nullptr;  // reciprocal pivots (node-block path)
    void spmv(const T* x, T* y, double* dot) const {
        PROF(FM_PROF_SPMV, 1);
        T* part = reinterpret_cast<T*>(c->partials.p);
        if (node_block)
            fm::launch_spmv_nodes<T>(c->nn, c->nbr_ptr.p, c->nbr.p, K, x, y, part, c->counter(),
                                     dot, c->stream);
        else
            fm::launch_spmv_csr<T>(S->n, S->rp.p, S->ci.p, K, x, y, part, c->counter(), dot,
                                   c->stream);
    }
    void precond(const T* r, T* z) const {
        const bool pu = node_block && (sizeof(T) == 4 ? c->pu_ok32 : c->pu_ok64);
        PROF(FM_PROF_TRSV, pu ? (r != z ? 3 : 4) : node_block ? 4 : 2);
        if (node_block) {
            precond_nodes<T>(c, LU, dinv, r, tmp, z, c->status());
            return;
        }
        const fm::CsrDev v = S->view();
        fm::launch_trsv_lower_csr<T>(v, LU, r, tmp, c->done.p, next_epoch(c), c->status(),
                                     grid_trsv, c->stream);
        fm::launch_trsv_upper_csr<T>(v, LU, diag, tmp, z, c->done.p, next_epoch(c), c->status(),
                                     grid_trsv, c->stream);
    }
};

// PCG-ILU(0) with the reference's stop tests (FEM/adaptive_fem_engine.hpp:1292-1340).
// b, x: length-n device vectors of type T; x in/out.
template <typename T>
fm_status pcg_core(fm_ctx* c, const Op<T>& A, uint32_t n, const T* b, T* x, double tol,
                   int max_iter, int* iters_out, double* relres_out) {
    Work<T>& w = work<T>(c);
    T* part = reinterpret_cast<T*>(c->partials.p);
    fm::DevScalars* sc = c->sc.p;
    CK(cudaMemsetAsync(&sc->stop, 0, sizeof(unsigned), c->stream));
    // r = b - A x
    A.spmv(x, w.r.p, nullptr);
    { PROF(FM_PROF_VECTOR, 1); fm::launch_residual_init<T>(n, b, w.r.p, part, c->counter(), &sc->rr, c->stream); }
    TRY(sync_scalars(c));
    TRY(check_flags(c, c->h_sc->status, "pcg"));
    int iters = max_iter;
    double relres = 0.0;
    if (std::sqrt(c->h_sc->rr) < tol * 1e-3) {
        iters = 0;
    } else {
        A.precond(w.r.p, w.z.p);
        { PROF(FM_PROF_VECTOR, 1); fm::launch_pcg_start<T>(n, w.r.p, w.z.p, b, w.p.p, part, c->counter(), sc, c->stream); }
        for (int it = 0; it < max_iter; ++it) {
            A.spmv(w.p.p, w.Ap.p, &sc->pAp);
            { PROF(FM_PROF_VECTOR, 1); fm::launch_pcg_update_xr<T>(n, w.p.p, w.Ap.p, x, w.r.p, sc, c->stream); }
            A.precond(w.r.p, w.z.p);
            { PROF(FM_PROF_VECTOR, 1); fm::launch_pcg_rz<T>(n, w.r.p, w.z.p, part, c->counter(), sc, c->stream); }
            TRY(sync_scalars(c));
            TRY(check_flags(c, c->h_sc->status, "pcg"));
            if (c->h_sc->stop) break;  // |p.Ap| < 1e-60
            relres = c->h_sc->relres;
            if (relres < tol) {
                iters = it + 1;
                break;
            }
            { PROF(FM_PROF_VECTOR, 1); fm::launch_pcg_update_p<T>(n, w.z.p, w.p.p, sc, c->stream); }
        }
    }
    if (iters_out) *iters_out = iters;
    if (relres_out) *relres_out = relres;
    return FM_OK;
}

template <typename T>
fm_status ilu_core(fm_ctx* c, SolverCsr& S, const T* a, T* lu, T* diag) {
    PROF(FM_PROF_ILU, &S == &c->fem ? 3 : 1);
    if (&S == &c->fem) {
        fm::launch_ilu0_nodes<T>(node_sched(c), a, lu, c->nnz, diag, work<T>(c).dinv.p,
                                 c->status(), c->device, c->stream);
        CK(cudaGetLastError());
        return FM_OK;
    }
    const fm::CsrDev v = S.view();
    const int grid = fm::persistent_grid_ilu0_csr(c->device, sizeof(T) == 4, v);
    fm::launch_ilu0_csr<T>(v, a, lu, diag, c->done.p, next_epoch(c), c->status(), grid,
                           c->stream);
    CK(cudaGetLastError());
    return FM_OK;
}

fm_status need_mesh(fm_ctx* c) {
    if (!c) return FM_ERR_ARG;
    if (!c->nn) return fail(c, FM_ERR_ARG, "no mesh: call fm_set_mesh first");
    return FM_OK;
}
fm_status need_material(fm_ctx* c) {
    TRY(need_mesh(c));
    if (!c->has_mat) return fail(c, FM_ERR_ARG, "no material: call fm_set_material first");
    return FM_OK;
}

template <typename T>
fm_status ensure_matrix(fm_ctx* c) {
    Work<T>& w = work<T>(c);
    CK(w.K.reserve(c->nnz));
    CK(w.LU.reserve(c->nnz));
    CK(w.diag.reserve(c->n));
    CK(w.dinv.reserve(c->n));
    return ensure_vectors<T>(c, c->n);
}

// DOF-level dependency levels of the solve pattern from the node levels:
// node n's rows hold all three DOFs of n and of each neighbour, so row 3n+d
// sits at depth 3 D(n) + d below and 3 D_U(n) + 2 - d above (D: node depth),
// and at depth 0 in both directions when n has no entries at all.  Rows of a
// level ascend, as a stable sort by depth orders them.
fm_status ensure_dof_levels(fm_ctx* c) {
    if (!c->lvl_fwd_ptr.empty() && !c->lvl_bwd_ptr.empty()) return FM_OK;
    const uint32_t nn = c->nn, n = c->n;
    for (int lower = 1; lower >= 0; --lower) {
        const std::vector<uint32_t>& lp = lower ? c->node_lp : c->node_up;
        const std::vector<uint32_t>& lo = lower ? c->node_lo : c->node_uo;
        std::vector<uint32_t> depth(n, 0);
        uint32_t maxd = 0;
        for (size_t l = 0; l + 1 < lp.size(); ++l)
            for (uint32_t t = lp[l]; t < lp[l + 1]; ++t) {
                const uint32_t nd = lo[t];
                if (c->graph.ptr[nd + 1] == c->graph.ptr[nd]) continue;  // no entries
                for (uint32_t d = 0; d < 3; ++d) {
                    const uint32_t dep = 3 * (uint32_t)l + (lower ? d : 2 - d);
                    depth[3 * nd + d] = dep;
                    maxd = std::max(maxd, dep);
                }
            }
        std::vector<uint32_t>& ptr = lower ? c->lvl_fwd_ptr : c->lvl_bwd_ptr;
        std::vector<uint32_t>& rows = lower ? c->lvl_fwd_rows : c->lvl_bwd_rows;
        const uint32_t nl = n ? maxd + 1 : 0;
        ptr.assign(nl + 1, 0);
        for (uint32_t i = 0; i < n; ++i) ptr[depth[i] + 1]++;
        for (uint32_t l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
        rows.resize(n);
        std::vector<uint32_t> fill(ptr.begin(), ptr.end() - (nl ? 1 : 0));
        for (uint32_t i = 0; i < n; ++i) rows[fill[depth[i]]++] = i;
    }
    (void)nn;
    return FM_OK;
}

// element -> CSR slot maps on the device (chunks of 2^20 tets through a
// scratch buffer): into host memory, or into a device buffer
fm_status slot_map_device(fm_ctx* c, int reference, int32_t* host_out, DevBuf<int32_t>* dev_out) {
    const uint32_t chunk = 1u << 20;
    DevBuf<int32_t> tmp;
    if (dev_out) CK(dev_out->reserve(144 * (size_t)std::max(c->ne, 1u)));
    else CK(tmp.reserve(144 * (size_t)std::min(c->ne, chunk)));
    for (uint32_t e0 = 0; e0 < c->ne; e0 += chunk) {
        const uint32_t cnt = std::min(chunk, c->ne - e0);
        int32_t* dst = dev_out ? dev_out->p + 144 * (size_t)e0 : tmp.p;
        fm::launch_slot_map(e0, cnt, c->conn.p, c->nbr_ptr.p, c->nbr.p, reference, dst,
                            c->stream);
        CK(cudaGetLastError());
        if (host_out)
            CK(cudaMemcpyAsync(host_out + 144 * (size_t)e0, dst, 144 * sizeof(int32_t) * cnt,
                               cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return FM_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

fm_status fm_create(fm_ctx** out, int device, void* stream) {
    if (!out) return FM_ERR_ARG;
    *out = nullptr;
    fm_ctx* c = nullptr;
    try {
        c = new fm_ctx;
    } catch (const std::bad_alloc&) {
        return FM_ERR_OOM;
    }
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete c;
        return FM_ERR_CUDA;
    }
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return FM_ERR_CUDA;
        }
        c->own_stream = true;
    }
    if (c->sc.reserve(1) != cudaSuccess || c->partials.reserve(8192) != cudaSuccess ||
        cudaMallocHost(&c->h_sc, sizeof(fm::DevScalars)) != cudaSuccess) {
        fm_destroy(c);
        return FM_ERR_OOM;
    }
    cudaMemsetAsync(c->sc.p, 0, sizeof(fm::DevScalars), c->stream);
    cudaMemsetAsync(c->partials.p, 0, c->partials.n * sizeof(double), c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        fm_destroy(c);
        return FM_ERR_CUDA;
    }
    c->grid_trsv64 = fm::persistent_grid_trsv_csr(device, false);
    c->grid_trsv32 = fm::persistent_grid_trsv_csr(device, true);
    *out = c;
    return FM_OK;
}

void fm_destroy(fm_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->h_sc) cudaFreeHost(c->h_sc);
    bool own = c->own_stream;
    cudaStream_t s = c->stream;
    delete c;
    if (own && s) cudaStreamDestroy(s);
}

fm_status fm_last_error(const fm_ctx* c, char* buf, size_t len) {
    if (!c || !buf || !len) return FM_ERR_ARG;
    std::snprintf(buf, len, "%s", c->err.c_str());
    return FM_OK;
}

fm_status fm_get_flags(fm_ctx* c, uint32_t* flags) {
    if (!c || !flags) return FM_ERR_ARG;
    return device_flags(c, flags);
}

fm_status fm_clear_flags(fm_ctx* c) {
    if (!c) return FM_ERR_ARG;
    CK(cudaMemsetAsync(&c->sc.p->status, 0, sizeof(unsigned), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FM_OK;
}

fm_status fm_set_wait_limit(fm_ctx* c, uint64_t cycles) {
    if (!c) return FM_ERR_ARG;
    const uint64_t units = (cycles + 1023) >> 10;
    if (units > 0xffffffffull) return fail(c, FM_ERR_ARG, "wait limit too large");
    c->h_sc->wait_budget = (unsigned)units;
    CK(cudaMemcpyAsync(&c->sc.p->wait_budget, &c->h_sc->wait_budget, sizeof(unsigned),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FM_OK;
}

fm_status fm_check_wait(fm_ctx* c) {
    if (!c) return FM_ERR_ARG;
    fm::launch_wait_probe(&c->sc.p->never, c->status(), c->stream);
    CK(cudaGetLastError());
    uint32_t flags;
    TRY(device_flags(c, &flags));
    return check_flags(c, flags, "fm_check_wait");
}

fm_status fm_sizes(const fm_ctx* c, uint32_t* n_nodes, uint32_t* n_elems, uint32_t* n_dofs,
                   uint64_t* nnz) {
    if (!c) return FM_ERR_ARG;
    if (n_nodes) *n_nodes = c->nn;
    if (n_elems) *n_elems = c->ne;
    if (n_dofs) *n_dofs = c->n;
    if (nnz) *nnz = c->nnz;
    return FM_OK;
}

fm_status fm_mesh_coloring(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn,
                           uint32_t* colors, uint32_t* n_colors) {
    if (!conn || !colors || !n_colors) return FM_ERR_ARG;
    for (size_t q = 0; q < 4 * (size_t)n_elems; ++q)
        if (conn[q] >= n_nodes) return FM_ERR_ARG;
    try {
        *n_colors = fm::mesh_coloring(n_nodes, n_elems, conn, colors);
    } catch (const std::bad_alloc&) {
        return FM_ERR_OOM;
    }
    return FM_OK;
}

fm_status fm_unit_cube_sizes(int N, uint32_t* n_nodes, uint32_t* n_elems) {
    if (N < 1 || N > 1200 || !n_nodes || !n_elems) return FM_ERR_ARG;
    const uint64_t s = (uint64_t)N + 1;
    *n_nodes = (uint32_t)(s * s * s);
    *n_elems = (uint32_t)(6ull * N * N * N);
    return FM_OK;
}

fm_status fm_unit_cube(int N, double* xyz, uint32_t* conn) {
    if (N < 1 || N > 1200 || !xyz || !conn) return FM_ERR_ARG;
    fm::unit_cube(N, xyz, conn);
    return FM_OK;
}

fm_status fm_set_mesh(fm_ctx* c, uint32_t n_nodes, const double* xyz, uint32_t n_elems,
                      const uint32_t* conn, const double* elem_volume) {
    if (!c) return FM_ERR_ARG;
    if (!xyz || !conn || !n_nodes || !n_elems) return fail(c, FM_ERR_ARG, "empty mesh");
    if (n_nodes >= (1u << 30)) return fail(c, FM_ERR_ARG, "n_nodes too large");
    try {
        CK(cudaSetDevice(c->device));
        // a new mesh starts with clear flags (a stale timeout would stop the
        // level pass's waits at once)
        CK(cudaMemsetAsync(&c->sc.p->status, 0, sizeof(unsigned), c->stream));
        for (size_t q = 0; q < 4 * (size_t)n_elems; ++q)
            if (conn[q] >= n_nodes)
                return fail(c, FM_ERR_ARG, "conn[%zu] = %u out of range", q, conn[q]);
        c->nn = n_nodes;
        c->ne = n_elems;
        c->n = 3 * n_nodes;
        c->h_xyz.assign(xyz, xyz + 3 * (size_t)n_nodes);
        c->h_conn.assign(conn, conn + 4 * (size_t)n_elems);
        c->h_skip.assign(n_elems, 0);
        if (elem_volume)
            for (uint32_t e = 0; e < n_elems; ++e) c->h_skip[e] = !(elem_volume[e] >= 1e-30);
        std::vector<uint4> cw(n_elems);
        for (uint32_t e = 0; e < n_elems; ++e) {
            const uint32_t* q = conn + 4 * (size_t)e;
            cw[e] = make_uint4(q[0] | (c->h_skip[e] ? 0x80000000u : 0u), q[1], q[2], q[3]);
        }
        CK(upload(c->xyz, xyz, 3 * (size_t)n_nodes, c->stream));
        CK(upload(c->conn, cw.data(), n_elems, c->stream));
        // incidence, node graph, dependency levels, ILU maps and the
        // assembly's scatter structure, built on the device
        fm::MeshSetupDev md{&c->inc_ptr,      &c->inc_e,    &c->nbr_ptr,  &c->nbr,
                            &c->self_pos,     &c->node_fwd, &c->node_bwd, &c->node_fwd_rec,
                            &c->node_bwd_rec, &c->emap_ptr, &c->emap,     &c->inc_pos,
                            &c->nbr_members};
        fm::MeshSetupHost mh;
        int res = fm::kSetupOk;
        CK(fm::build_mesh_device(n_nodes, n_elems, c->conn.p, md, mh, c->status(), &res,
                                 c->stream));
        if (res == fm::kSetupTimeout)
            return fail(c, FM_ERR_TIMEOUT, "fm_set_mesh: a bounded wait of the level pass expired");
        if (res == fm::kSetupLimits)
            return fail(c, FM_ERR_LIMITS,
                        "mesh valence beyond kernel limits (max neighbours %u, max incident "
                        "tets %u; both must be <= 32)",
                        mh.graph.max_deg, mh.max_inc);
        c->graph = std::move(mh.graph);
        const uint64_t nnz = 9ull * c->graph.ptr[n_nodes];
        if (nnz >= (1ull << 32)) return fail(c, FM_ERR_LIMITS, "nnz %llu exceeds 32-bit CSR",
                                             (unsigned long long)nnz);
        c->nnz = nnz;
        // the scalar CSR and its DOF-level levels are built on first use
        // (fm_build_pattern, fm_levels): the node kernels never read them
        c->fem.n = c->n;
        c->fem.nnz = nnz;
        c->fem.h_rp.clear();
        c->fem.h_ci.clear();
        c->lvl_fwd_ptr.clear();
        c->lvl_bwd_ptr.clear();
        c->node_lp = std::move(mh.lp);
        c->node_lo = std::move(mh.lo);
        c->node_up = std::move(mh.up);
        c->node_uo = std::move(mh.uo);
        c->node_levels_fwd = (uint32_t)c->node_lp.size() - 1;
        c->node_levels_bwd = (uint32_t)c->node_up.size() - 1;
        c->width_fwd = c->width_bwd = 0;
        for (size_t l = 0; l + 1 < c->node_lp.size(); ++l)
            c->width_fwd = std::max(c->width_fwd, c->node_lp[l + 1] - c->node_lp[l]);
        for (size_t l = 0; l + 1 < c->node_up.size(); ++l)
            c->width_bwd = std::max(c->width_bwd, c->node_up[l + 1] - c->node_up[l]);
        TRY(setup_push_solves(c, c->node_lp, c->node_lo, c->node_up, c->node_uo));
        CK(cudaStreamSynchronize(c->stream));
        CK(c->done.reserve(std::max<size_t>(c->done.n, (size_t)c->nn + 1)));
        CK(cudaMemsetAsync(c->done.p, 0, c->done.n * sizeof(unsigned), c->stream));
        c->w64.factor_valid = c->w32.factor_valid = false;
        c->has_bc = false;
        c->has_mat = false;
        c->ref_slot.release();
        CK(c->vec_a.reserve(c->n));
        CK(c->vec_b.reserve(c->n));
        CK(c->elem_rec.reserve(std::max<size_t>(1, (size_t)c->ne * fm::kElemRecBytes)));
        CK(cudaStreamSynchronize(c->stream));
    } catch (const std::bad_alloc&) {
        return fail(c, FM_ERR_OOM, "host allocation failed in fm_set_mesh");
    }
    return FM_OK;
}

fm_status fm_build_pattern(fm_ctx* c, fm_pattern kind, uint32_t* row_ptr_out,
                           uint32_t* col_idx_out, int32_t* slot_map_out) {
    TRY(need_mesh(c));
    try {
        if (kind != FM_PATTERN_REFERENCE && kind != FM_PATTERN_SOLVE)
            return fail(c, FM_ERR_ARG, "unknown pattern kind %d", (int)kind);
        if (row_ptr_out) {
            row_ptr_out[0] = 0;
            fm::csr_row_ptr(c->graph, row_ptr_out);
        }
        if (col_idx_out) {
            if (kind == FM_PATTERN_REFERENCE) fm::csr_reference_cols(c->graph, col_idx_out);
            else fm::csr_solve_cols(c->graph, col_idx_out);
        }
        if (slot_map_out)
            TRY(slot_map_device(c, kind == FM_PATTERN_REFERENCE, slot_map_out, nullptr));
    } catch (const std::bad_alloc&) {
        return fail(c, FM_ERR_OOM, "host allocation failed in fm_build_pattern");
    }
    return FM_OK;
}

fm_status fm_set_material(fm_ctx* c, double E, double nu, const double* E_elem) {
    TRY(need_mesh(c));
    if (!(nu > -1.0 && nu < 0.5)) return fail(c, FM_ERR_ARG, "nu must be in (-1, 0.5)");
    c->nu = nu;
    // mu, lambda exactly as the reference forms them (FEM/adaptive_fem_engine.hpp:81-82)
    c->mu_s = E / (2.0 * (1.0 + nu));
    c->lam_s = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    c->c_mu = 1.0 / (2.0 * (1.0 + nu));
    c->c_lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double one_m = 1.0 - 2.0 * nu;
    c->inv_cnu = 1.0 / (one_m < 0.1 ? 0.1 : one_m);
    if (E_elem) {
        CK(upload(c->m0, E_elem, c->ne, c->stream));
        c->mat_mode = 1;
    } else {
        c->mat_mode = 0;
    }
    CK(cudaStreamSynchronize(c->stream));
    c->has_mat = true;
    return FM_OK;
}

fm_status fm_set_material_lame(fm_ctx* c, const double* mu_elem, const double* lambda_elem,
                               double nu) {
    TRY(need_mesh(c));
    if (!mu_elem || !lambda_elem) return fail(c, FM_ERR_ARG, "mu/lambda arrays required");
    if (!(nu > -1.0 && nu < 0.5)) return fail(c, FM_ERR_ARG, "nu must be in (-1, 0.5)");
    c->nu = nu;
    const double one_m = 1.0 - 2.0 * nu;
    c->inv_cnu = 1.0 / (one_m < 0.1 ? 0.1 : one_m);
    CK(upload(c->m0, mu_elem, c->ne, c->stream));
    CK(upload(c->m1, lambda_elem, c->ne, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->mat_mode = 2;
    c->has_mat = true;
    return FM_OK;
}

fm_status fm_set_bc(fm_ctx* c, const uint8_t* dof_mask, const double* dof_value) {
    TRY(need_mesh(c));
    if (!dof_mask) {
        c->has_bc = false;
        return FM_OK;
    }
    std::vector<uint8_t> m(dof_mask, dof_mask + c->n);
    for (auto& v : m) v = v ? 1 : 0;
    CK(upload(c->mask, m.data(), c->n, c->stream));
    c->has_bcval = dof_value != nullptr;
    if (dof_value) CK(upload(c->bcval, dof_value, c->n, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->has_bc = true;
    return FM_OK;
}

fm_status fm_elements(fm_ctx* c, uint32_t n, const double* x, const double* u, const double* E,
                      double nu, double* K, double* f) {
    if (!c || !x || !u || !E || !K || !f) return fail(c, FM_ERR_ARG, "null argument");
    { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_elements(n, x, u, E, nu, K, f, c->status(), c->stream); }
    CK(cudaGetLastError());
    uint32_t flags;
    TRY(device_flags(c, &flags));
    return check_flags(c, flags, "fm_elements");
}

fm_status fm_assemble(fm_ctx* c, const double* u, void* K, double* f, fm_precision prec,
                      int apply_bc) {
    TRY(need_material(c));
    if (!u) return fail(c, FM_ERR_ARG, "u is null");
    const fm::MeshDev m = mesh_view(c);
    if (prec == FM_FP64) {
        TRY(ensure_matrix<double>(c));
        double* Kd = K ? static_cast<double*>(K) : c->w64.K.p;
        { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, Kd, f, nullptr, apply_bc && c->has_bc, c->status(), c->stream); }
        c->w64.factor_valid = false;
    } else if (prec == FM_MIXED) {
        TRY(ensure_matrix<float>(c));
        float* Kf = K ? static_cast<float*>(K) : c->w32.K.p;
        { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, Kf, f, nullptr, apply_bc && c->has_bc, c->status(), c->stream); }
        c->w32.factor_valid = false;
    } else {
        return fail(c, FM_ERR_ARG, "unknown precision");
    }
    CK(cudaGetLastError());
    return FM_OK;
}

fm_status fm_assemble_host(fm_ctx* c, const double* u_host, double* K_host, double* f_host) {
    TRY(need_material(c));
    if (!u_host) return fail(c, FM_ERR_ARG, "u is null");
    TRY(ensure_matrix<double>(c));
    CK(cudaMemcpyAsync(c->vec_a.p, u_host, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                       c->stream));
    const fm::MeshDev m = mesh_view(c);
    { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, c->vec_a.p, c->w64.K.p, c->vec_b.p, nullptr, 0, c->status(),
                        c->stream); }
    CK(cudaGetLastError());
    c->w64.factor_valid = false;
    if (K_host)
        CK(cudaMemcpyAsync(K_host, c->w64.K.p, sizeof(double) * c->nnz, cudaMemcpyDeviceToHost,
                           c->stream));
    if (f_host)
        CK(cudaMemcpyAsync(f_host, c->vec_b.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                           c->stream));
    uint32_t flags;
    TRY(device_flags(c, &flags));
    return check_flags(c, flags, "fm_assemble_host");
}

fm_status fm_residual(fm_ctx* c, const double* u, double* f) {
    TRY(need_material(c));
    if (!u || !f) return fail(c, FM_ERR_ARG, "null argument");
    const fm::MeshDev m = mesh_view(c);
    { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, static_cast<double*>(nullptr), f, nullptr, 0, c->status(),
                        c->stream); }
    CK(cudaGetLastError());
    return FM_OK;
}

fm_status fm_assemble_reference_pattern(fm_ctx* c, const double* u, double* K, double* f) {
    TRY(need_material(c));
    if (!u || !K || !f) return fail(c, FM_ERR_ARG, "null argument");
    if (!c->ref_slot.p) TRY(slot_map_device(c, 1, nullptr, &c->ref_slot));
    CK(c->ke_scratch.reserve(144 * (size_t)c->ne));
    CK(cudaMemsetAsync(K, 0, sizeof(double) * c->nnz, c->stream));
    CK(cudaMemsetAsync(f, 0, sizeof(double) * c->n, c->stream));
    { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble_slotmap(mesh_view(c), u, c->ref_slot.p, K, f, c->ke_scratch.p,
                                c->status(), c->stream); }
    CK(cudaGetLastError());
    uint32_t flags;
    TRY(device_flags(c, &flags));
    return check_flags(c, flags, "fm_assemble_reference_pattern");
}

fm_status fm_levels(fm_ctx* c, uint32_t* fwd_ptr, uint32_t* fwd_rows, uint32_t* bwd_ptr,
                    uint32_t* bwd_rows, uint32_t* n_fwd, uint32_t* n_bwd) {
    TRY(need_mesh(c));
    try {
        TRY(ensure_dof_levels(c));
    } catch (const std::bad_alloc&) {
        return fail(c, FM_ERR_OOM, "host allocation failed in fm_levels");
    }
    if (fwd_ptr) std::copy(c->lvl_fwd_ptr.begin(), c->lvl_fwd_ptr.end(), fwd_ptr);
    if (fwd_rows) std::copy(c->lvl_fwd_rows.begin(), c->lvl_fwd_rows.end(), fwd_rows);
    if (bwd_ptr) std::copy(c->lvl_bwd_ptr.begin(), c->lvl_bwd_ptr.end(), bwd_ptr);
    if (bwd_rows) std::copy(c->lvl_bwd_rows.begin(), c->lvl_bwd_rows.end(), bwd_rows);
    if (n_fwd) *n_fwd = (uint32_t)c->lvl_fwd_ptr.size() - 1;
    if (n_bwd) *n_bwd = (uint32_t)c->lvl_bwd_ptr.size() - 1;
    return FM_OK;
}

fm_status fm_ilu0(fm_ctx* c, fm_precision prec) {
    TRY(need_mesh(c));
    if (prec == FM_FP64) {
        TRY(ensure_matrix<double>(c));
        TRY(ilu_core<double>(c, c->fem, c->w64.K.p, c->w64.LU.p, c->w64.diag.p));
        c->w64.factor_valid = true;
    } else if (prec == FM_MIXED) {
        TRY(ensure_matrix<float>(c));
        TRY(ilu_core<float>(c, c->fem, c->w32.K.p, c->w32.LU.p, c->w32.diag.p));
        c->w32.factor_valid = true;
    } else {
        return fail(c, FM_ERR_ARG, "unknown precision");
    }
    uint32_t flags;
    TRY(device_flags(c, &flags));
    return check_flags(c, flags, "fm_ilu0");
}

fm_status fm_get_ilu0(fm_ctx* c, double* LU, double* diag) {
    TRY(need_mesh(c));
    if (!c->w64.factor_valid) return fail(c, FM_ERR_ARG, "no FP64 factorization: call fm_ilu0");
    if (LU)
        CK(cudaMemcpyAsync(LU, c->w64.LU.p, sizeof(double) * c->nnz, cudaMemcpyDeviceToHost,
                           c->stream));
    if (diag)
        CK(cudaMemcpyAsync(diag, c->w64.diag.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                           c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FM_OK;
}

fm_status fm_ilu0_apply(fm_ctx* c, const double* r, double* y) {
    TRY(need_mesh(c));
    if (!c->w64.factor_valid) return fail(c, FM_ERR_ARG, "no FP64 factorization: call fm_ilu0");
    if (!r || !y) return fail(c, FM_ERR_ARG, "null argument");
    Op<double> A{c, &c->fem, true, c->w64.K.p, c->w64.LU.p, c->w64.diag.p, c->w64.t.p,
                 c->grid_trsv64, c->w64.dinv.p};
    A.precond(r, y);
    CK(cudaGetLastError());
    uint32_t flags;
    TRY(device_flags(c, &flags));
    return check_flags(c, flags, "fm_ilu0_apply");
}

// ---- fm_ilu0_apply_noalloc ------------------------------------------------
// For callers that must not allocate device memory during the call: the
// intermediate z = L^-1 r of the two node-block solves and the status word
// of their bounded waits live in this file-scope array instead of context
// buffers.  One array per device for the whole process (8 MiB + 256 B, held
// until exit); every context on the device shares it, so calls that overlap
// on the GPU race on it.
struct NoAllocScratch {
    double z[FM_NOALLOC_MAX_DOFS];
    unsigned status;
    unsigned wait_budget;  // the calling context's wait limit (read after status)
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kNoAllocMaxDevices = 64;

// Device address of g_noalloc_scratch, looked up once per device with that
// device current (the caller's current device is restored afterwards).  The
// lookup may load the module.  (Host code must never pass g_noalloc_scratch
// itself to a kernel: on the host that name is a stand-in, not a device
// address.)
static fm_status noalloc_scratch(fm_ctx* c, NoAllocScratch** out) {
    static std::mutex mu;
    static NoAllocScratch* addr[kNoAllocMaxDevices] = {};
    if (c->device < 0 || c->device >= kNoAllocMaxDevices)
        return fail(c, FM_ERR_LIMITS, "fm_ilu0_apply_noalloc: device %d beyond %d", c->device,
                    kNoAllocMaxDevices);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[c->device]) {
        int prev = 0;
        CK(cudaGetDevice(&prev));
        CK(cudaSetDevice(c->device));
        NoAllocScratch* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        CK(cudaSetDevice(prev));
        CK(e);
        addr[c->device] = ptr;
    }
    *out = addr[c->device];
    return FM_OK;
}

fm_status fm_ilu0_apply_noalloc(fm_ctx* c, const double* r, double* y) {
    TRY(need_mesh(c));
    if (c->n > FM_NOALLOC_MAX_DOFS)
        return fail(c, FM_ERR_LIMITS,
                    "fm_ilu0_apply_noalloc: %u DOFs exceed the scratch limit of %u DOFs", c->n,
                    (unsigned)FM_NOALLOC_MAX_DOFS);
    if (!c->w64.factor_valid) return fail(c, FM_ERR_ARG, "no FP64 factorization: call fm_ilu0");
    if (!r || !y) return fail(c, FM_ERR_ARG, "null argument");
    NoAllocScratch* sp = nullptr;
    TRY(noalloc_scratch(c, &sp));
    // the status word keeps the previous call's bits: it must start at zero;
    // the wait limit is this context's; z is refilled with the wait sentinel
    // by the launcher before each solve
    CK(cudaMemsetAsync(&sp->status, 0, sizeof(unsigned), c->stream));
    CK(cudaMemcpyAsync(&sp->wait_budget, &c->sc.p->wait_budget, sizeof(unsigned),
                       cudaMemcpyDeviceToDevice, c->stream));
    precond_nodes<double>(c, c->w64.LU.p, c->w64.dinv.p, r, sp->z, y, &sp->status);
    CK(cudaGetLastError());
    unsigned flags = 0;
    CK(cudaMemcpyAsync(&flags, &sp->status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return check_flags(c, flags, "fm_ilu0_apply_noalloc");
}

fm_status fm_spmv(fm_ctx* c, const double* x, double* y) {
    TRY(need_mesh(c));
    if (!x || !y || !c->w64.K.p) return fail(c, FM_ERR_ARG, "null argument or no K");
    Op<double> A{c, &c->fem, true, c->w64.K.p, nullptr, nullptr, nullptr, 0};
    A.spmv(x, y, nullptr);
    CK(cudaGetLastError());
    return FM_OK;
}

fm_status fm_pcg(fm_ctx* c, const double* b, double* x, double tol, int max_iter, int* iters,
                 double* relres, fm_precision prec) {
    TRY(need_mesh(c));
    if (!b || !x || max_iter < 0) return fail(c, FM_ERR_ARG, "bad argument");
    if (prec == FM_FP64) {
        if (!c->w64.factor_valid) return fail(c, FM_ERR_ARG, "call fm_ilu0(FM_FP64) first");
        Op<double> A{c, &c->fem, true, c->w64.K.p, c->w64.LU.p, c->w64.diag.p, c->w64.t.p,
                     c->grid_trsv64, c->w64.dinv.p};
        return pcg_core<double>(c, A, c->n, b, x, tol, max_iter, iters, relres);
    }
    if (prec != FM_MIXED) return fail(c, FM_ERR_ARG, "unknown precision");
    if (!c->w32.factor_valid) return fail(c, FM_ERR_ARG, "call fm_ilu0(FM_MIXED) first");
    // FP32 inner solve on b/||b||; x returned in FP64
    { PROF(FM_PROF_VECTOR, 1); fm::launch_norm2(c->n, b, c->partials.p, c->counter(), &c->sc.p->norm2, c->stream); }
    TRY(sync_scalars(c));
    const double s = std::sqrt(c->h_sc->norm2);
    if (s == 0.0) {
        if (iters) *iters = 0;
        if (relres) *relres = 0.0;
        return FM_OK;
    }
    { PROF(FM_PROF_VECTOR, 1); fm::launch_to_f32_scaled(c->n, b, 1.0 / s, c->w32.b.p, c->w32.x.p, c->stream); }
    Op<float> A{c, &c->fem, true, c->w32.K.p, c->w32.LU.p, c->w32.diag.p, c->w32.t.p,
                c->grid_trsv32, c->w32.dinv.p};
    TRY(pcg_core<float>(c, A, c->n, c->w32.b.p, c->w32.x.p, tol, max_iter, iters, relres));
    { PROF(FM_PROF_VECTOR, 1); fm::launch_axpy_u_f32(c->n, c->w32.x.p, s, x, c->stream); }
    CK(cudaGetLastError());
    return FM_OK;
}

fm_status fm_csr_pcg_ilu0(fm_ctx* c, uint32_t n, const uint32_t* row_ptr,
                          const uint32_t* col_idx, const double* val, const double* b,
                          double* x, double tol, int max_iter, int* iters, double* relres) {
    if (!c || !row_ptr || !col_idx || !val || !b || !x || n == 0)
        return fail(c, FM_ERR_ARG, "bad argument");
    try {
        const uint64_t nnz = row_ptr[n];
        // sort columns per row (values follow), as the reference's symbolic
        // phase sorts its L/U patterns
        std::vector<uint32_t> rp(row_ptr, row_ptr + n + 1), ci(col_idx, col_idx + nnz);
        std::vector<double> v(val, val + nnz);
        std::vector<std::pair<uint32_t, double>> row;
        for (uint32_t i = 0; i < n; ++i) {
            if (rp[i + 1] < rp[i] || rp[i + 1] > nnz)
                return fail(c, FM_ERR_ARG, "row_ptr not monotone at row %u", i);
            row.clear();
            for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
                if (ci[k] >= n) return fail(c, FM_ERR_ARG, "column %u out of range", ci[k]);
                row.emplace_back(ci[k], v[k]);
            }
            std::stable_sort(row.begin(), row.end(),
                             [](const auto& a, const auto& b2) { return a.first < b2.first; });
            for (size_t q = 0; q < row.size(); ++q) {
                ci[rp[i] + q] = row[q].first;
                v[rp[i] + q] = row[q].second;
            }
        }
        if (c->gen.n != n || c->gen.h_rp != rp || c->gen.h_ci != ci)
            TRY(setup_solver_csr(c, c->gen, n, std::move(rp), std::move(ci)));
        CK(upload(c->gen_K, v.data(), nnz, c->stream));
        CK(c->gen_LU.reserve(nnz));
        CK(c->gen_diag.reserve(n));
        TRY(ensure_vectors<double>(c, n));
        CK(c->vec_a.reserve(n));
        CK(c->vec_b.reserve(n));
        CK(cudaMemcpyAsync(c->vec_a.p, b, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->vec_b.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
        TRY(ilu_core<double>(c, c->gen, c->gen_K.p, c->gen_LU.p, c->gen_diag.p));
        Op<double> A{c, &c->gen, false, c->gen_K.p, c->gen_LU.p, c->gen_diag.p, c->w64.t.p,
                     c->grid_trsv64};
        TRY(pcg_core<double>(c, A, n, c->vec_a.p, c->vec_b.p, tol, max_iter, iters, relres));
        CK(cudaMemcpyAsync(x, c->vec_b.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    } catch (const std::bad_alloc&) {
        return fail(c, FM_ERR_OOM, "host allocation failed");
    }
    return FM_OK;
}

fm_status fm_newton_config_default(fm_newton_config* g) {
    if (!g) return FM_ERR_ARG;
    g->newton_rtol = 1e-10;
    g->newton_atol = 0.0;
    g->inner_tol = 1e-12;
    g->predictor_tol = 0.0;
    g->inner_tol_min = 0.0;
    g->max_newton = 200;
    g->max_pcg = 5000;
    g->line_search = 10;
    g->ls_c = 1e-4;
    g->diverge_rate = 0.0;
    g->diverge_count = 3;
    g->diverge_growth = 10.0;
    g->precision = FM_FP64;
    g->ilu_every = 1;
    g->initial_guess = 0;
    return FM_OK;
}

fm_status fm_newton_step_cfg(fm_ctx* c, double* u, double load_frac, const fm_newton_config* g,
                             fm_newton_result* res) {
    if (res) std::memset(res, 0, sizeof *res);
    TRY(need_material(c));
    if (!u || !g || g->max_newton < 1 || g->line_search < 0 || g->max_pcg < 1 ||
        !(g->inner_tol > 0.0) || g->ilu_every < 1)
        return fail(c, FM_ERR_ARG, "bad argument");
    const int prec = g->precision;
    if (prec != FM_FP64 && prec != FM_MIXED) return fail(c, FM_ERR_ARG, "unknown precision");
    const bool mixed = prec == FM_MIXED;
    if (mixed) TRY(ensure_matrix<float>(c));
    else TRY(ensure_matrix<double>(c));
    CK(c->vec_c.reserve(c->n));
    CK(c->vec_d.reserve(c->n));
    const fm::MeshDev m = mesh_view(c);
    double* R = c->vec_a.p;
    double* du = c->vec_b.p;
    const bool keep_du = g->line_search > 0;
    int n_newton = 0, n_pcg = 0, n_bt = 0, slow = 0;
    double r0 = 0.0, rn = 0.0, r_prev = 0.0;
    double tol = g->inner_tol;
    bool have_r0 = false;
    fm_status out = FM_OK;
    c->newton_hist.clear();
    auto record = [&](int kind, int its, double rnorm, double alpha, double itol) {
        if (c->newton_hist.size() < 4096)
            c->newton_hist.push_back({kind, its, rnorm, alpha, itol, c->h_sc->status, 0u});
    };

    // ILU(0) of the eliminated tangent, PCG on R (norm rnorm) to itol, then
    // either u += du or du kept in `du` (FP64) for the line search.
    int n_solve = 0;
    bool have_prev = false;  // w32.x holds the previous Newton correction / ||R||
    auto solve = [&](double rnorm, double itol, bool keep, int* its, bool newton) -> fm_status {
        const bool refactor = n_solve++ % g->ilu_every == 0;
        if (mixed) {
            // FP32 tangent/ILU(0)/PCG on R/||R||; the step is rescaled in FP64
            if (refactor) TRY(ilu_core<float>(c, c->fem, c->w32.K.p, c->w32.LU.p, c->w32.diag.p));
            const bool guess = g->initial_guess && newton && have_prev;
            { PROF(FM_PROF_VECTOR, 1); fm::launch_to_f32_scaled(c->n, R, 1.0 / rnorm, c->w32.b.p, guess ? nullptr : c->w32.x.p, c->stream); }
            if (guess) {
                // x0 = gamma x_prev with gamma = x_prev.b / x_prev.K x_prev: the
                // energy-norm projection of the solution on the previous
                // correction (corrections of a linearly converging Newton
                // iteration are nearly parallel); never worse than x0 = 0
                float* part = reinterpret_cast<float*>(c->partials.p);
                {
                    PROF(FM_PROF_SPMV, 1);
                    fm::launch_spmv_nodes<float>(c->nn, c->nbr_ptr.p, c->nbr.p, c->w32.K.p,
                                                 c->w32.x.p, c->w32.Ap.p, nullptr, nullptr,
                                                 nullptr, c->stream);
                }
                {
                    PROF(FM_PROF_VECTOR, 2);
                    fm::launch_dot<float>(c->n, c->w32.x.p, c->w32.b.p, part, c->counter(),
                                          &c->sc.p->guess_xb, c->stream);
                    fm::launch_dot<float>(c->n, c->w32.x.p, c->w32.Ap.p, part, c->counter(),
                                          &c->sc.p->guess_xkx, c->stream);
                }
                TRY(sync_scalars(c));
                const double xkx = c->h_sc->guess_xkx;
                const double gam = xkx > 0.0 && std::isfinite(xkx) ? c->h_sc->guess_xb / xkx : 0.0;
                { PROF(FM_PROF_VECTOR, 1); fm::launch_scale_f32(c->n, c->w32.x.p, (float)gam, c->stream); }
            }
            Op<float> A{c, &c->fem, true, c->w32.K.p, c->w32.LU.p, c->w32.diag.p, c->w32.t.p,
                        c->grid_trsv32, c->w32.dinv.p};
            TRY(pcg_core<float>(c, A, c->n, c->w32.b.p, c->w32.x.p, itol, g->max_pcg, its,
                                nullptr));
            if (keep) { PROF(FM_PROF_VECTOR, 1); fm::launch_f32_to_f64_scaled(c->n, c->w32.x.p, rnorm, du, c->stream); }
            else { PROF(FM_PROF_VECTOR, 1); fm::launch_axpy_u_f32(c->n, c->w32.x.p, rnorm, u, c->stream); }
            have_prev = newton;
        } else {
            if (refactor) TRY(ilu_core<double>(c, c->fem, c->w64.K.p, c->w64.LU.p, c->w64.diag.p));
            CK(cudaMemsetAsync(du, 0, sizeof(double) * c->n, c->stream));
            Op<double> A{c, &c->fem, true, c->w64.K.p, c->w64.LU.p, c->w64.diag.p, c->w64.t.p,
                         c->grid_trsv64, c->w64.dinv.p};
            TRY(pcg_core<double>(c, A, c->n, R, du, itol, g->max_pcg, its, nullptr));
            if (!keep) { PROF(FM_PROF_VECTOR, 1); fm::launch_axpy_u(c->n, du, u, c->stream); }
        }
        CK(cudaGetLastError());
        return FM_OK;
    };

    // the engine updates the element states after every Newton update of u
    // (FEM/adaptive_fem_engine.hpp:2589); here when state arrays are attached
    auto update_states = [&]() {
        if (!c->state_F || !c->state_stress) return;
        PROF(FM_PROF_STATES, 1);
        fm::launch_element_states(m, u, c->nu, c->state_F, c->state_stress,
                                  c->sc.p->state_counts, c->stream);
    };

    auto finish = [&](fm_status st) -> fm_status {
        c->w64.factor_valid = c->w32.factor_valid = false;
        if (res) {
            res->newton_iters = n_newton;
            res->pcg_iters = n_pcg;
            res->backtracks = n_bt;
            res->flags = c->h_sc->status;
            res->rnorm0 = r0;
            res->rnorm = rn;
            res->final_relres = r0 > 0 ? rn / r0 : 0.0;
        }
        return st;
    };

    if (c->has_bc) {
        // predictor: spread the prescribed increment v through the body with
        // the tangent at the current state (K_ff du_f = -f_f - K_fc v_c)
        double* v = c->vec_d.p;
        { PROF(FM_PROF_VECTOR, 1); fm::launch_bc_increment(c->n, c->mask.p, c->has_bcval ? c->bcval.p : nullptr, load_frac,
                                u, v, mixed ? c->w32.b.p : nullptr, c->partials.p, c->counter(),
                                &c->sc.p->norm2, c->stream); }
        TRY(sync_scalars(c));
        if (c->h_sc->norm2 > 0.0) {
            double* f = c->vec_c.p;
            if (mixed) {
                { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, c->w32.K.p, f, nullptr, 0, c->status(), c->stream); }
                { PROF(FM_PROF_SPMV, 1); fm::launch_spmv_nodes<float>(c->nn, c->nbr_ptr.p, c->nbr.p, c->w32.K.p,
                                             c->w32.b.p, c->w32.Ap.p, nullptr, nullptr, nullptr,
                                             c->stream); }
                { PROF(FM_PROF_VECTOR, 1); fm::launch_predictor_rhs<float>(c->n, c->mask.p, f, c->w32.Ap.p, R, c->stream); }
                { PROF(FM_PROF_VECTOR, 1); fm::launch_apply_bc_nodes<float>(c->nn, c->nbr_ptr.p, c->nbr.p, c->mask.p,
                                                 c->w32.K.p, c->stream); }
            } else {
                { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, c->w64.K.p, f, nullptr, 0, c->status(), c->stream); }
                { PROF(FM_PROF_SPMV, 1); fm::launch_spmv_nodes<double>(c->nn, c->nbr_ptr.p, c->nbr.p, c->w64.K.p, v,
                                              c->w64.Ap.p, nullptr, nullptr, nullptr, c->stream); }
                { PROF(FM_PROF_VECTOR, 1); fm::launch_predictor_rhs<double>(c->n, c->mask.p, f, c->w64.Ap.p, R, c->stream); }
                { PROF(FM_PROF_VECTOR, 1); fm::launch_apply_bc_nodes<double>(c->nn, c->nbr_ptr.p, c->nbr.p, c->mask.p,
                                                  c->w64.K.p, c->stream); }
            }
            { PROF(FM_PROF_VECTOR, 1); fm::launch_norm2(c->n, R, c->partials.p, c->counter(), &c->sc.p->norm2, c->stream); }
            TRY(sync_scalars(c));
            if (fm_status st = check_flags(c, c->h_sc->status, "newton predictor")) return finish(st);
            r0 = rn = std::sqrt(c->h_sc->norm2);
            have_r0 = true;
            int its = 0;
            const double ptol = g->predictor_tol > 0.0 ? g->predictor_tol : tol;
            if (r0 > 0.0) TRY(solve(r0, ptol, false, &its, false));
            n_pcg += its;
            ++n_newton;
            record(0, its, r0, 1.0, ptol);
            r_prev = r0;
        }
        { PROF(FM_PROF_VECTOR, 1); fm::launch_set_bc_values(c->n, c->mask.p, c->has_bcval ? c->bcval.p : nullptr, load_frac,
                                 u, c->stream); }
        update_states();
    }

    bool conv = false;
    for (int it = n_newton; it < g->max_newton; ++it) {
        if (mixed)
            { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, c->w32.K.p, nullptr, R, 1, c->status(), c->stream); }
        else
            { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, u, c->w64.K.p, nullptr, R, 1, c->status(), c->stream); }
        { PROF(FM_PROF_VECTOR, 1); fm::launch_norm2(c->n, R, c->partials.p, c->counter(), &c->sc.p->norm2, c->stream); }
        TRY(sync_scalars(c));
        rn = std::sqrt(c->h_sc->norm2);
        if (fm_status st = check_flags(c, c->h_sc->status, "newton assembly")) {
            record(1, 0, rn, 0.0, tol);
            return finish(fail(c, st, "%s; Newton iteration %d of load %.6g, ||R|| history "
                                      "(last): %.3e",
                               c->err.c_str(), it, load_frac, r_prev));
        }
        if (!have_r0) {
            r0 = rn;
            have_r0 = true;
        }
        if (rn == 0.0 || rn < g->newton_rtol * r0 || rn < g->newton_atol) {
            conv = true;
            record(1, 0, rn, 0.0, tol);
            break;
        }
        // the reference's divergence test (FEM/adaptive_fem_engine.hpp:2561-2572)
        if (it > 2) {
            const double rate = rn / std::max(r_prev, 1e-30);
            if (g->diverge_rate > 0.0 && rate > g->diverge_rate) ++slow;
            if ((g->diverge_rate > 0.0 && slow > g->diverge_count) ||
                (g->diverge_growth > 0.0 && rn > r_prev * g->diverge_growth)) {
                record(1, 0, rn, 0.0, tol);
                return finish(fail(c, FM_ERR_DIVERGED,
                                   "Newton diverging at iteration %d of load %.6g: ||R|| %.3e "
                                   "(previous %.3e, ||R_0|| %.3e, slow iterations %d; flags: %s)",
                                   it, load_frac, rn, r_prev, r0, slow,
                                   flags_text(c->h_sc->status).c_str()));
            }
        }
        // adaptive inner tolerance: an iteration that did not contract by
        // diverge_rate (0.9 when the rate test is off) tightens the next solves
        if (g->inner_tol_min > 0.0 && r_prev > 0.0 &&
            rn > (g->diverge_rate > 0.0 ? g->diverge_rate : 0.9) * r_prev)
            tol = std::max(g->inner_tol_min, 0.1 * tol);
        int its = 0;
        TRY(solve(rn, tol, keep_du, &its, true));
        double alpha = 1.0;
        if (keep_du) {
            // Armijo backtracking on ||R|| with residual-only re-assembly at
            // each trial point (armijo_line_search_true, :933-985)
            // flags raised at rejected trial points (a clamped or non-finite
            // trial) are dropped: the accepted state's next assembly decides
            const unsigned status0 = c->h_sc->status;
            for (int bt = 0; bt < g->line_search; ++bt) {
                { PROF(FM_PROF_VECTOR, 1); fm::launch_trial(c->n, u, alpha, du, c->vec_c.p, c->stream); }
                { PROF(FM_PROF_ASSEMBLE, 1); fm::launch_assemble(m, c->vec_c.p, static_cast<double*>(nullptr), nullptr, R, 0,
                                    c->status(), c->stream); }
                { PROF(FM_PROF_VECTOR, 1); fm::launch_norm2(c->n, R, c->partials.p, c->counter(), &c->sc.p->norm2,
                                 c->stream); }
                TRY(sync_scalars(c));
                const double rt = std::sqrt(c->h_sc->norm2);
                if (rt <= (1.0 - g->ls_c * alpha) * rn + 1e-14) break;
                alpha *= 0.5;
                ++n_bt;
            }
            { PROF(FM_PROF_VECTOR, 1); fm::launch_trial(c->n, u, alpha, du, u, c->stream); }
            c->h_sc->status = status0;
            CK(cudaMemcpyAsync(&c->sc.p->status, &c->h_sc->status, sizeof(unsigned),
                               cudaMemcpyHostToDevice, c->stream));
            TRY(sync_scalars(c));
        }
        CK(cudaGetLastError());
        update_states();
        n_pcg += its;
        ++n_newton;
        record(1, its, rn, alpha, tol);
        r_prev = rn;
    }
    CK(cudaStreamSynchronize(c->stream));
    if (!conv) {
        TRY(sync_scalars(c));
        return finish(fail(c, FM_ERR_NOT_CONVERGED,
                           "Newton hit max_newton=%d at load %.6g (||R||/||R_0|| = %.3e; flags: %s)",
                           g->max_newton, load_frac, r0 > 0 ? rn / r0 : 0.0,
                           flags_text(c->h_sc->status).c_str()));
    }
    return finish(out);
}

fm_status fm_element_states(fm_ctx* c, const double* u, double* F, double* stress,
                            uint32_t* det_violations, uint32_t* nonfinite) {
    TRY(need_material(c));
    if (!u || !F || !stress) return fail(c, FM_ERR_ARG, "null argument");
    CK(cudaMemsetAsync(c->sc.p->state_counts, 0, 2 * sizeof(unsigned), c->stream));
    {
        PROF(FM_PROF_STATES, 1);
        fm::launch_element_states(mesh_view(c), u, c->nu, F, stress, c->sc.p->state_counts,
                                  c->stream);
    }
    CK(cudaGetLastError());
    TRY(sync_scalars(c));
    if (det_violations) *det_violations = c->h_sc->state_counts[0];
    if (nonfinite) *nonfinite = c->h_sc->state_counts[1];
    return FM_OK;
}

fm_status fm_set_state_output(fm_ctx* c, double* F, double* stress) {
    TRY(need_mesh(c));
    if ((F == nullptr) != (stress == nullptr))
        return fail(c, FM_ERR_ARG, "give both state arrays or neither");
    c->state_F = F;
    c->state_stress = stress;
    return FM_OK;
}

fm_status fm_newton_history(const fm_ctx* c, fm_newton_record* out, int cap, int* count) {
    if (!c || !count || cap < 0 || (cap > 0 && !out)) return FM_ERR_ARG;
    const int n = (int)std::min<size_t>(c->newton_hist.size(), (size_t)cap);
    for (int i = 0; i < n; ++i) out[i] = c->newton_hist[i];
    *count = (int)c->newton_hist.size();
    return FM_OK;
}

fm_status fm_newton_step(fm_ctx* c, double* u, double load_frac, double rtol, double atol,
                         double inner_tol, int max_newton, int max_pcg, int line_search,
                         double ls_c, fm_precision prec, int* newton_iters, int* pcg_iters,
                         double* final_relres) {
    fm_newton_config g;
    fm_newton_config_default(&g);
    g.newton_rtol = rtol;
    g.newton_atol = atol;
    g.inner_tol = inner_tol;
    g.max_newton = max_newton;
    g.max_pcg = max_pcg;
    g.line_search = line_search;
    g.ls_c = ls_c;
    g.precision = prec;
    fm_newton_result r;
    const fm_status st = fm_newton_step_cfg(c, u, load_frac, &g, &r);
    if (newton_iters) *newton_iters = r.newton_iters;
    if (pcg_iters) *pcg_iters = r.pcg_iters;
    if (final_relres) *final_relres = r.final_relres;
    return st;
}

fm_status fm_newton_solve_cfg(fm_ctx* c, double* u, int first_step, int n_steps,
                              const fm_newton_config* cfg, fm_newton_result* result) {
    if (result) std::memset(result, 0, sizeof *result);
    TRY(need_material(c));
    if (!u || !cfg || n_steps < 1 || first_step < 1 || first_step > n_steps)
        return fail(c, FM_ERR_ARG, "bad load-step range");
    fm_newton_result tot;
    std::memset(&tot, 0, sizeof tot);
    fm_status worst = FM_OK;
    for (int s = first_step; s <= n_steps; ++s) {
        fm_newton_result r;
        const fm_status st = fm_newton_step_cfg(c, u, (double)s / (double)n_steps, cfg, &r);
        tot.newton_iters += r.newton_iters;
        tot.pcg_iters += r.pcg_iters;
        tot.backtracks += r.backtracks;
        tot.flags = r.flags;
        tot.rnorm0 = r.rnorm0;
        tot.rnorm = r.rnorm;
        tot.final_relres = r.final_relres;
        if (result) *result = tot;
        if (st == FM_ERR_NOT_CONVERGED) worst = st;
        else if (st != FM_OK) return st;
    }
    if (worst != FM_OK)
        return fail(c, worst, "a load step hit max_newton=%d", cfg->max_newton);
    return FM_OK;
}

fm_status fm_newton_solve(fm_ctx* c, double* u, int first_step, int n_steps, double rtol,
                          double atol, double inner_tol, int max_newton, int max_pcg,
                          fm_precision prec, int* newton_iters, int* pcg_iters,
                          double* final_relres) {
    fm_newton_config g;
    fm_newton_config_default(&g);
    g.newton_rtol = rtol;
    g.newton_atol = atol;
    g.inner_tol = inner_tol;
    g.max_newton = max_newton;
    g.max_pcg = max_pcg;
    g.precision = prec;
    fm_newton_result r;
    const fm_status st = fm_newton_solve_cfg(c, u, first_step, n_steps, &g, &r);
    if (newton_iters) *newton_iters = r.newton_iters;
    if (pcg_iters) *pcg_iters = r.pcg_iters;
    if (final_relres) *final_relres = r.final_relres;
    return st;
}

fm_status fm_csr_ilu0(fm_ctx* c, uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                      const double* val, double* LU_out, double* diag_out) {
    if (!c || !row_ptr || !col_idx || !val || n == 0) return fail(c, FM_ERR_ARG, "bad argument");
    try {
        const uint64_t nnz = row_ptr[n];
        std::vector<uint32_t> rp(row_ptr, row_ptr + n + 1), ci(col_idx, col_idx + nnz);
        std::vector<double> v(val, val + nnz);
        std::vector<uint32_t> perm(nnz);  // sorted slot -> caller slot
        for (uint32_t i = 0; i < n; ++i) {
            if (rp[i + 1] < rp[i] || rp[i + 1] > nnz)
                return fail(c, FM_ERR_ARG, "row_ptr not monotone at row %u", i);
            for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
                if (col_idx[k] >= n) return fail(c, FM_ERR_ARG, "column out of range");
                perm[k] = k;
            }
            std::stable_sort(perm.begin() + rp[i], perm.begin() + rp[i + 1],
                             [&](uint32_t a, uint32_t b) { return col_idx[a] < col_idx[b]; });
            for (uint32_t k = rp[i]; k < rp[i + 1]; ++k) {
                ci[k] = col_idx[perm[k]];
                v[k] = val[perm[k]];
            }
        }
        if (c->gen.n != n || c->gen.h_rp != rp || c->gen.h_ci != ci)
            TRY(setup_solver_csr(c, c->gen, n, std::move(rp), std::move(ci)));
        CK(upload(c->gen_K, v.data(), nnz, c->stream));
        CK(c->gen_LU.reserve(nnz));
        CK(c->gen_diag.reserve(n));
        TRY(ilu_core<double>(c, c->gen, c->gen_K.p, c->gen_LU.p, c->gen_diag.p));
        std::vector<double> lu(nnz);
        CK(cudaMemcpyAsync(lu.data(), c->gen_LU.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost,
                           c->stream));
        if (diag_out)
            CK(cudaMemcpyAsync(diag_out, c->gen_diag.p, sizeof(double) * n,
                               cudaMemcpyDeviceToHost, c->stream));
        uint32_t flags;
        TRY(device_flags(c, &flags));
        TRY(check_flags(c, flags, "fm_csr_ilu0"));
        if (LU_out)
            for (uint64_t k = 0; k < nnz; ++k) LU_out[perm[k]] = lu[k];
    } catch (const std::bad_alloc&) {
        return fail(c, FM_ERR_OOM, "host allocation failed");
    }
    return FM_OK;
}

fm_status fm_newton_step_host(fm_ctx* c, double* u_host, double load_frac, double rtol,
                              double atol, double inner_tol, int max_newton, int max_pcg,
                              int line_search, double ls_c, fm_precision prec, int* newton_iters,
                              int* pcg_iters, double* final_relres) {
    TRY(need_mesh(c));
    if (!u_host) return fail(c, FM_ERR_ARG, "u is null");
    CK(c->vec_e.reserve(c->n));
    CK(cudaMemcpyAsync(c->vec_e.p, u_host, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                       c->stream));
    fm_status st = fm_newton_step(c, c->vec_e.p, load_frac, rtol, atol, inner_tol, max_newton,
                                  max_pcg, line_search, ls_c, prec, newton_iters, pcg_iters,
                                  final_relres);
    if (st != FM_OK && st != FM_ERR_NOT_CONVERGED) return st;
    CK(cudaMemcpyAsync(u_host, c->vec_e.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return st;
}

fm_status fm_newton_step_cfg_host(fm_ctx* c, double* u_host, double load_frac,
                                  const fm_newton_config* cfg, fm_newton_result* result) {
    TRY(need_mesh(c));
    if (!u_host) return fail(c, FM_ERR_ARG, "u is null");
    CK(c->vec_e.reserve(c->n));
    CK(cudaMemcpyAsync(c->vec_e.p, u_host, sizeof(double) * c->n, cudaMemcpyHostToDevice,
                       c->stream));
    const fm_status st = fm_newton_step_cfg(c, c->vec_e.p, load_frac, cfg, result);
    if (st != FM_OK && st != FM_ERR_NOT_CONVERGED) return st;
    CK(cudaMemcpyAsync(u_host, c->vec_e.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return st;
}

fm_status fm_profile_enable(fm_ctx* c, int on) {
    if (!c) return FM_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    prof_flush(c);
    for (int k = 0; k < FM_PROF_KINDS; ++k) {
        c->prof_ms[k] = 0.0;
        c->prof_calls[k] = c->prof_kernels[k] = 0;
    }
    c->prof_on = on != 0;
    return FM_OK;
}

fm_status fm_profile_read(fm_ctx* c, fm_profile* out) {
    if (!c || !out) return FM_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    prof_flush(c);
    for (int k = 0; k < FM_PROF_KINDS; ++k) {
        out->ms[k] = c->prof_ms[k];
        out->calls[k] = c->prof_calls[k];
        out->kernels[k] = c->prof_kernels[k];
    }
    return FM_OK;
}

fm_status fm_exact_apply(fm_ctx* c, const double* u, const double* v, double* y, int transpose) {
    TRY(need_material(c));
    if (!u || !v || !y) return fail(c, FM_ERR_ARG, "null argument");
    {
        PROF(FM_PROF_ASSEMBLE, 1);
        fm::launch_exact_apply(mesh_view(c), u, v, y, transpose ? 1 : 0, c->stream);
    }
    CK(cudaGetLastError());
    return FM_OK;
}

// Adjoint by defect correction: the exact Jacobian K is non-symmetric, the
// reference tangent K_t (symmetric, with its ILU(0)) is the preconditioner:
//   w <- w + PCG(K_t, g - K^T w)   on the free DOFs, until
//   ||g - K^T w|| <= tol ||g||.
// FM_MIXED runs K_t, its ILU(0) and the PCG in FP32 on the scaled defect;
// K^T w, the defect and w stay FP64, so the sweeps restore FP64 accuracy.
fm_status fm_adjoint(fm_ctx* c, const double* u, const double* dLdu, double* gmu, double* glam,
                     double* w_out, double tol, double inner_tol, int max_sweeps,
                     fm_precision prec, int* sweeps_out, int* pcg_out) {
    TRY(need_material(c));
    if (!u || !dLdu || !gmu || !glam || max_sweeps < 1)
        return fail(c, FM_ERR_ARG, "bad argument");
    if (prec != FM_FP64 && prec != FM_MIXED) return fail(c, FM_ERR_ARG, "unknown precision");
    const bool mixed = prec == FM_MIXED;
    if (mixed) TRY(ensure_matrix<float>(c));
    else TRY(ensure_matrix<double>(c));
    CK(c->vec_c.reserve(c->n));
    CK(c->vec_d.reserve(c->n));
    CK(c->vec_e.reserve(c->n));
    const fm::MeshDev m = mesh_view(c);
    const uint8_t* mask = c->has_bc ? c->mask.p : nullptr;
    double* w = w_out ? w_out : c->vec_e.p;
    double* r = c->vec_a.p;
    double* dw = c->vec_b.p;
    double* y = c->vec_c.p;
    // preconditioner: reference tangent at u, eliminated, and its ILU(0)
    {
        PROF(FM_PROF_ASSEMBLE, 1);
        if (mixed) fm::launch_assemble(m, u, c->w32.K.p, nullptr, nullptr, 1, c->status(), c->stream);
        else fm::launch_assemble(m, u, c->w64.K.p, nullptr, nullptr, 1, c->status(), c->stream);
    }
    if (mixed) TRY(ilu_core<float>(c, c->fem, c->w32.K.p, c->w32.LU.p, c->w32.diag.p));
    else TRY(ilu_core<double>(c, c->fem, c->w64.K.p, c->w64.LU.p, c->w64.diag.p));
    CK(cudaMemsetAsync(w, 0, sizeof(double) * c->n, c->stream));
    // ||g|| on the free DOFs
    CK(cudaMemsetAsync(y, 0, sizeof(double) * c->n, c->stream));
    {
        PROF(FM_PROF_VECTOR, 1);
        fm::launch_adj_residual(c->n, mask, dLdu, y, r, c->partials.p, c->counter(),
                                &c->sc.p->norm2, c->stream);
    }
    TRY(sync_scalars(c));
    const double gn = std::sqrt(c->h_sc->norm2);
    int sweeps = 0, pcg_total = 0;
    bool conv = gn == 0.0;
    double rn = gn;
    for (; !conv && sweeps < max_sweeps; ++sweeps) {
        int its = 0;
        if (mixed) {
            {
                PROF(FM_PROF_VECTOR, 1);
                fm::launch_to_f32_scaled(c->n, r, 1.0 / rn, c->w32.b.p, c->w32.x.p, c->stream);
            }
            Op<float> A{c, &c->fem, true, c->w32.K.p, c->w32.LU.p, c->w32.diag.p, c->w32.t.p,
                        c->grid_trsv32, c->w32.dinv.p};
            TRY(pcg_core<float>(c, A, c->n, c->w32.b.p, c->w32.x.p, inner_tol, 100000, &its,
                                nullptr));
            {
                PROF(FM_PROF_VECTOR, 1);
                fm::launch_f32_to_f64_scaled(c->n, c->w32.x.p, rn, dw, c->stream);
            }
        } else {
            CK(cudaMemsetAsync(dw, 0, sizeof(double) * c->n, c->stream));
            Op<double> A{c, &c->fem, true, c->w64.K.p, c->w64.LU.p, c->w64.diag.p, c->w64.t.p,
                         c->grid_trsv64, c->w64.dinv.p};
            TRY(pcg_core<double>(c, A, c->n, r, dw, inner_tol, 100000, &its, nullptr));
        }
        pcg_total += its;
        {
            PROF(FM_PROF_VECTOR, 1);
            fm::launch_adj_update(c->n, mask, dw, w, c->stream);
        }
        {
            PROF(FM_PROF_ASSEMBLE, 1);
            fm::launch_exact_apply(m, u, w, y, 1, c->stream);
        }
        {
            PROF(FM_PROF_VECTOR, 1);
            fm::launch_adj_residual(c->n, mask, dLdu, y, r, c->partials.p, c->counter(),
                                    &c->sc.p->norm2, c->stream);
        }
        TRY(sync_scalars(c));
        TRY(check_flags(c, c->h_sc->status, "fm_adjoint"));
        rn = std::sqrt(c->h_sc->norm2);
        if (rn <= tol * gn) conv = true;
    }
    {
        PROF(FM_PROF_ASSEMBLE, 1);
        fm::launch_param_grads(m, u, w, gmu, glam, c->stream);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    c->w64.factor_valid = c->w32.factor_valid = false;
    if (sweeps_out) *sweeps_out = sweeps;
    if (pcg_out) *pcg_out = pcg_total;
    if (!conv)
        return fail(c, FM_ERR_NOT_CONVERGED, "adjoint: %d sweeps, defect %.3e of %.3e", sweeps,
                    rn, gn);
    return FM_OK;
}

}  // extern "C"
