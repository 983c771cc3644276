// C ABI of the B200 HDG element hot path (declared in include/hfem_b200.h).
//
// Host side of the library: context and device buffers, connectivity checks,
// kernel dispatch over the compiled element shapes, GMRES and the Newton
// driver (restating solvers/dgsolvers.cpp:40-205).  Every entry point returns
// a status code; nothing exits the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <queue>
#include <string>
#include <vector>

#include "../../include/hfem_b200.h"
#include "elem_kernels.cuh"
#include "krylov_kernels.cuh"
#include "krylov_seg.cuh"
#include "schur_kernels.cuh"
#include "elem_kernel.cuh"
#include "lift.cuh"
#include "schur_tc.cuh"
#include "bilu0.cuh"
#include "inverse_blocked.cuh"
#include "schur_fused.cuh"

using namespace hfem;

namespace {

constexpr int RNORM_CTAS = 296;

struct KernelTimer {
    bool on = false;
    std::map<std::string, std::pair<double, int>> acc;
    std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
};

// Element shapes with compiled kernels: (nd, npv, npf, ngv, ngf).
#define HFEM_SHAPES(X)          \
    X(2, 3, 2, 3, 2)            \
    X(2, 6, 3, 6, 3)            \
    X(2, 10, 4, 12, 4)          \
    X(2, 15, 5, 16, 5)          \
    X(3, 4, 3, 4, 3)            \
    X(3, 10, 6, 14, 6)          \
    X(3, 20, 10, 24, 12)

// GEMM tile choices per shape (m-tiles, n-tiles per warp, warps): g1 for D^-1 F
// (n x nb, K = n), g2 for H - K D^-1 F (nb x nb, K = n); the fastest of the
// candidates below on a B200, timed on 20k-51k-element meshes of each shape.
// Small CTAs (1-3 warps, 2-stage) win: many resident CTAs hide the short
// (K <= 100) main loops' fill and drain.
template <class S> struct SchurCfg;
template <> struct SchurCfg<Shape<2, 3, 2, 3, 2>> { using g1 = GemmCfg<2, 3, 1>; using g2 = GemmCfg<3, 3, 1>; };
template <> struct SchurCfg<Shape<2, 6, 3, 6, 3>> { using g1 = GemmCfg<3, 5, 1>; using g2 = GemmCfg<5, 3, 2>; };
template <> struct SchurCfg<Shape<2, 10, 4, 12, 4>> { using g1 = GemmCfg<5, 3, 2>; using g2 = GemmCfg<6, 3, 2>; };
template <> struct SchurCfg<Shape<2, 15, 5, 16, 5>> { using g1 = GemmCfg<4, 4, 2>; using g2 = GemmCfg<4, 2, 4>; };
template <> struct SchurCfg<Shape<3, 4, 3, 4, 3>> { using g1 = GemmCfg<3, 4, 2>; using g2 = GemmCfg<4, 2, 4>; };
template <> struct SchurCfg<Shape<3, 10, 6, 14, 6>> { using g1 = GemmCfg<4, 4, 2>; using g2 = GemmCfg<4, 2, 4>; };
template <> struct SchurCfg<Shape<3, 20, 10, 24, 12>> { using g1 = GemmCfg<5, 3, 3>; using g2 = GemmCfg<5, 3, 2>; };

struct GemmLaunch {
    int bm, bn, threads;
    size_t smem;
    const void* fn;
    void (*run)(cudaStream_t, int, int, int, int, double, const double*, int, long long, const double*, int,
                long long, double, double*, int, long long);
};

template <class G, int MT, int WN, int NW, int BK, int ST>
void run_gemm(cudaStream_t st, int batch, int M, int N, int K, double alpha, const double* A, int lda, long long sA,
              const double* B, int ldb, long long sB, double beta, double* C, int ldc, long long sC) {
    const int tiles = ((M + G::BM - 1) / G::BM) * ((N + G::BN - 1) / G::BN);
    batched_dgemm_kernel<MT, WN, NW, BK, ST><<<(unsigned)(tiles * batch), G::THREADS, G::SMEM, st>>>(
        M, N, K, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC);
}

template <class G> struct GemmParams;
template <int MT, int WN, int NW, int BK, int ST> struct GemmParams<GemmCfg<MT, WN, NW, BK, ST>> {
    static GemmLaunch make() {
        using G = GemmCfg<MT, WN, NW, BK, ST>;
        return GemmLaunch{G::BM, G::BN, G::THREADS, G::SMEM, (const void*)batched_dgemm_kernel<MT, WN, NW, BK, ST>,
                          run_gemm<G, MT, WN, NW, BK, ST>};
    }
};

// Every batched-GEMM tiling compiled into the library; any of them is valid
// for any shape (edges are masked), so the autotuner may pick any.
const std::vector<GemmLaunch>& gemm_candidates() {
    static std::vector<GemmLaunch> v = {
        GemmParams<GemmCfg<2, 3, 1>>::make(), GemmParams<GemmCfg<3, 3, 1>>::make(),
        GemmParams<GemmCfg<3, 5, 1>>::make(), GemmParams<GemmCfg<5, 5, 1>>::make(),
        GemmParams<GemmCfg<5, 3, 2>>::make(), GemmParams<GemmCfg<6, 3, 2>>::make(),
        GemmParams<GemmCfg<4, 4, 2>>::make(), GemmParams<GemmCfg<3, 4, 2>>::make(),
        GemmParams<GemmCfg<7, 3, 5>>::make(), GemmParams<GemmCfg<5, 3, 5>>::make(),
        GemmParams<GemmCfg<5, 5, 5>>::make(), GemmParams<GemmCfg<4, 2, 4>>::make(),
        GemmParams<GemmCfg<5, 4, 2>>::make(), GemmParams<GemmCfg<5, 3, 3>>::make(),
        GemmParams<GemmCfg<5, 5, 5, 12, 4>>::make(), GemmParams<GemmCfg<5, 3, 2, 20, 3>>::make(),
    };
    return v;
}

struct Launch {
    int nd, npv, npf, ngv, ngf;
    size_t ws;                  // workspace doubles per CTA slot (element_kernel)
    size_t q_smem;
    void (*getq)(dim3, size_t, cudaStream_t, const QArgs&);
    void (*inverse)(dim3, cudaStream_t, int, double*, const double*, double*, int*);
    void (*element)(dim3, size_t, cudaStream_t, const ElemArgs&);
    // [tf][gen]: 3xTF32 contractions; Lax-Friedrichs / Roe tensor or Sutherland's law compiled in
    void (*element_v[2][2])(dim3, size_t, cudaStream_t, const ElemArgs&);
    size_t elem_smem;
    const void* elem_fn;
    const void* elem_fn_v[2][2];
    int inv_threads;
    size_t inv_smem;
    const void *q_fn, *inv_fn;
    GemmLaunch g1, g2;
    void (*schur_tc)(dim3, size_t, cudaStream_t, const SchurTcArgs&);
    size_t tc_smem;
    int tc_tmem;                // tensor-memory columns of one tensor-core Schur CTA
    const void* tc_fn;
    void (*scatter_h)(dim3, cudaStream_t, const ScatterArgs&);
    void (*schur_fused)(cudaStream_t, int, const double*, const double*, const double*, double*, double*);
    size_t fused_smem;
    const void* fused_fn;
};

template <int N>
void launch_inverse(dim3 g, cudaStream_t st, int ne, double* D, const double* Ru, double* RuOut, int* info) {
    inverse_blocked_kernel<N><<<g, InvBlk<N>::THREADS, InvBlk<N>::SMEM, st>>>(ne, D, Ru, RuOut, info);
}

template <class S, bool TF, bool GEN>
void launch_element(dim3 g, size_t sm, cudaStream_t st, const ElemArgs& a) {
    element_kernel<S, TF, GEN><<<g, NT, sm, st>>>(a);
}
template <class S>
void launch_getq(dim3 g, size_t sm, cudaStream_t st, const QArgs& a) { getq_kernel<S><<<g, NT, sm, st>>>(a); }
template <class S>
void launch_scatter_h(dim3 g, cudaStream_t st, const ScatterArgs& a) {
    scatter_H_block_kernel<S::NPF, S::NCH, S::NFE><<<g, 256, 0, st>>>(a);
}
template <class S>
void launch_schur_tc(dim3 g, size_t sm, cudaStream_t st, const SchurTcArgs& a) {
    schur_tc_kernel<S::N, S::NB><<<g, TC_THREADS, sm, st>>>(a);
}

// strip width and warps of the fused FP64 condensation per shape
template <class S>
struct FusedPick {
    static constexpr int BN = S::NB >= 40 ? 40 : ((S::NB + 7) / 8) * 8;
    static constexpr int MT = (S::N + 7) / 8;
    static constexpr int NW = MT >= 4 ? 4 : MT;
    using Cfg = FusedCfg<S::N, S::NB, BN, NW>;
};
template <class S>
void launch_schur_fused(cudaStream_t st, int ne, const double* Dinv, const double* F, const double* K, double* H,
                        double* DinvF) {
    static_assert(S::NB <= LIFT_MAXNB, "the lift stages one column of H per warp");
    using P = FusedPick<S>;
    schur_fused_kernel<S::N, S::NB, P::BN, P::NW>
        <<<(unsigned)(ne * P::Cfg::STRIPS), P::Cfg::THREADS, P::Cfg::SMEM, st>>>(ne, Dinv, F, K, H, DinvF);
}

template <class S>
Launch make_launch() {
    Launch L;
    L.nd = S::ND; L.npv = S::NPV; L.npf = S::NPF; L.ngv = S::NGV; L.ngf = S::NGF;
    L.ws = EK<S>::WS;
    L.q_smem = sizeof(QSmem<S>);
    L.getq = launch_getq<S>;
    L.q_fn = (const void*)getq_kernel<S>;
    L.inverse = launch_inverse<S::N>;
    L.element = launch_element<S, false, false>;
    L.element_v[0][0] = launch_element<S, false, false>;
    L.element_v[0][1] = launch_element<S, false, true>;
    L.element_v[1][0] = launch_element<S, true, false>;
    L.element_v[1][1] = launch_element<S, true, true>;
    L.elem_smem = sizeof(ElemSmem<S>);
    L.elem_fn = (const void*)element_kernel<S, false, false>;
    L.elem_fn_v[0][0] = (const void*)element_kernel<S, false, false>;
    L.elem_fn_v[0][1] = (const void*)element_kernel<S, false, true>;
    L.elem_fn_v[1][0] = (const void*)element_kernel<S, true, false>;
    L.elem_fn_v[1][1] = (const void*)element_kernel<S, true, true>;
    L.inv_threads = InvBlk<S::N>::THREADS;
    L.inv_smem = InvBlk<S::N>::SMEM;
    L.inv_fn = (const void*)inverse_blocked_kernel<S::N>;
    L.g1 = GemmParams<typename SchurCfg<S>::g1>::make();
    L.g2 = GemmParams<typename SchurCfg<S>::g2>::make();
    L.schur_tc = launch_schur_tc<S>;
    L.tc_smem = TcCfg<S::N, S::NB>::SMEM;
    L.tc_tmem = (int)TcCfg<S::N, S::NB>::TMEM_COLS;
    L.tc_fn = (const void*)schur_tc_kernel<S::N, S::NB>;
    L.scatter_h = launch_scatter_h<S>;
    L.schur_fused = launch_schur_fused<S>;
    L.fused_smem = FusedPick<S>::Cfg::SMEM;
    L.fused_fn = (const void*)schur_fused_kernel<S::N, S::NB, FusedPick<S>::BN, FusedPick<S>::NW>;
    return L;
}

const std::vector<Launch>& launches() {
    static std::vector<Launch> v = {
#define X(a, b, c, d, e) make_launch<Shape<a, b, c, d, e>>(),
        HFEM_SHAPES(X)
#undef X
    };
    return v;
}

}  // namespace

struct hfem_ctx {
    hfem_dims dims{};
    int device = 0;
    int ncu = 0, nc = 0, nch = 0, ndf = 0, n = 0, nb = 0, bsz = 0;
    const Launch* L = nullptr;
    cudaStream_t own = nullptr, stream = nullptr;
    std::string err;
    bool have_master = false, have_mesh = false, have_phys = false, have_sol = false, assembled = false;
    int grid_elem = 0, grid_inv = 0, grid_tc = 0;
    int grid_elem_v[2][2] = {};         // per element-kernel variant [tf][gen], at most grid_elem
    // element-wise state arriving in pieces (hfem_assemble_host): the element
    // kernel of piece k waits for chunk_ev[k]
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> chunk_ev;
    std::vector<int> chunk_lo;              // first element of each piece, plus ne
    int pending_chunks = 0;
    double* seg_partk = nullptr;            // CGS2 partial dots, npieces x (restart + 1)
    size_t seg_partk_n = 0;
    int seg_hP = 0;
    // 0 FP64; 1 3xTF32 element contractions, TF32 tensor-core Schur GEMMs, FP32
    // preconditioner; 2 FP32 preconditioner only; 3 3xTF32 element contractions,
    // FP64 Schur, FP32 preconditioner
    int precision = 0;
    int g1_sel = -1, g2_sel = -1;   // autotuned batched-GEMM tilings (-1: the shape's default)
    // boundary faces (mesh.bf, app.bcm, app.bcs); bf == NULL: no boundary faces
    int *bf = nullptr, *bcm = nullptr;
    double* bcs = nullptr;
    int nbnd = 0;
    int appname = 1;            // app.appname: 1 Navier-Stokes, 0 Euler
    int conv_stab = 0;          // app.convStabMethod: 0 constant tau, 1 Lax-Friedrichs, 2 Roe
    int visc_model = 0;         // app.viscosityModel: 0 constant, 1 Sutherland's law
    int* tc_err = nullptr;              // 1: a tcgen05 MMA wait expired; 2: an element bulk-copy wait expired
    double* rn_part = nullptr;
    // master tables
    double *shapvt = nullptr, *shapvg = nullptr, *svsv = nullptr, *shapft = nullptr, *shapfg = nullptr, *sfsf = nullptr;
    int* perm = nullptr;
    // mesh
    double* dgnodes = nullptr;
    int *elcon = nullptr, *rowstart = nullptr, *colidx = nullptr, *blk_src = nullptr, *face_src = nullptr;
    int *rowface = nullptr, *colface = nullptr;
    std::vector<int> h_rowstart, h_colidx;
    // physics
    double param[6] = {0};
    int tdep = 0;
    double fc_u = 0, fc_q = 1, time = 0;
    // state
    double *udg = nullptr, *uh = nullptr, *sh = nullptr;
    // assembly outputs and workspace
    double *D = nullptr, *F = nullptr, *K = nullptr, *H = nullptr, *Ru = nullptr, *Rh = nullptr, *Ro = nullptr;
    double* DinvRu = nullptr;           // D^-1 Ru of the last matrix pass (the update's input)
    double* DinvF = nullptr;
    double *ru2 = nullptr, *Hg = nullptr, *Rg = nullptr, *Rr = nullptr, *rnorm = nullptr, *ws = nullptr;
    int* info = nullptr;
    // Krylov
    double *Minv = nullptr, *V = nullptr, *w = nullptr, *x = nullptr, *pb = nullptr, *scal = nullptr, *part = nullptr;
    float* Minv32 = nullptr;    // FP32 block-Jacobi inverses (mixed mode)
    int* binfo = nullptr;
    int krylov_restart = 0;
    double* udgi = nullptr;     // state at the start of the current time step
    // several problems in one mesh
    int nprob = 0;
    bool palpha_on = false;
    int *eprob = nullptr, *fprob = nullptr;
    double *pparam = nullptr, *palpha = nullptr;
    // per-problem Krylov segments (faces of each problem contiguous)
    int npieces = 0;
    long long* seg_pstart = nullptr;
    int *seg_pseg = nullptr, *seg_p0 = nullptr, *seg_ticket = nullptr;
    double *seg_part = nullptr, *seg_h = nullptr, *seg_y = nullptr, *seg_nrm = nullptr;
    // GMRES bookkeeping on the device (GmState): Hessenberg, rotations, g, rhs norms, states
    double *gm_H = nullptr, *gm_cs = nullptr, *gm_sn = nullptr, *gm_g = nullptr, *gm_nrmb = nullptr, *gm_hist = nullptr;
    int *gm_state = nullptr, *gm_its = nullptr, *gm_jc = nullptr;
    size_t gm_hist_n = 0;
    unsigned char* seg_act = nullptr;
    int* seg_k = nullptr;
    int seg_restart = 0;
    bool seg_single = false;    // segment tables describe one segment over the whole vector
    // BILU0: ordering (computed once, from the first system), level schedule, factors
    bool have_order = false;
    std::vector<int> h_o2u, h_u2o, lvl_lo, lvl_up;
    int *d_u2o = nullptr, *d_rows_lo = nullptr, *d_rows_up = nullptr, *d_fptr = nullptr, *d_fpos = nullptr;
    // flattened per-slot lists of the one-CTA factorisation and solves (BiluSched)
    int *d_frec = nullptr, *d_lrec = nullptr, *d_urec = nullptr;
    bool bilu_sched = false;            // the one-CTA factorisation and solves apply (BiluSched)
    int bilu_nslot_lo = 0, bilu_nslot_up = 0;   // slot-table rows of the one-CTA solves
    int *d_lvl_lo = nullptr, *d_lvl_up = nullptr;
    cudaGraphExec_t bilu_exec = nullptr;    // the factorisation's per-level launches, replayed as one graph
    double *Mg = nullptr, *bl_t = nullptr, *bl_y = nullptr;
    float* Mg32 = nullptr;              // FP32 copy of the BILU0 factors (mixed precision)
    int prec_kind = 2;                  // preconditioner of the current GMRES: 2 BJ, 0 BILU0, -1 none
    KernelTimer timer;
};

namespace {

int fail(hfem_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(c, HFEM_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Device memory of contexts comes from a per-process pool of size-class
// blocks: the buffers of a destroyed context are kept and handed to the next
// context that asks for the same class, so building and dropping contexts
// (the serving loop repacks them at iteration boundaries) does not pay
// cudaMalloc / cudaFree, each of which synchronises the device.  A block is
// returned to the pool only after its context's stream is idle.
// hfem_pool_trim gives the cached blocks back to the driver; a failed
// cudaMalloc trims and retries once.
struct DevicePool {
    std::mutex m;
    std::mutex trim;                                              // held while cached blocks are released
    std::map<std::pair<int, size_t>, std::vector<void*>> free;   // (device, class) -> idle blocks
    std::map<void*, std::pair<int, size_t>> live;                // block -> (device, class)
    std::map<int, size_t> cached_on;                              // device -> idle bytes
    std::map<int, size_t> cap;                                    // device -> most idle bytes kept
    size_t cached = 0;
};

DevicePool& pool() {
    static DevicePool* p = new DevicePool();        // outlives every context (never destroyed)
    return *p;
}

size_t size_class(size_t bytes) {
    if (bytes <= 256) return 256;
    if (bytes <= (1u << 20)) {
        size_t s = 256;
        while (s < bytes) s <<= 1;
        return s;
    }
    const size_t step = 2u << 20;
    return (bytes + step - 1) / step * step;
}

// Releases the idle blocks of one device (all devices: -1).  The releases run
// under P.trim, so a thread whose allocation failed while another thread was
// releasing waits for those releases before it retries.
size_t pool_trim_device(int device) {
    DevicePool& P = pool();
    std::lock_guard<std::mutex> t(P.trim);
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> g(P.m);
        for (auto it = P.free.begin(); it != P.free.end();) {
            if (device < 0 || it->first.first == device) {
                for (void* q : it->second) drop.push_back(q);
                const size_t b = it->first.second * it->second.size();
                P.cached -= b;
                P.cached_on[it->first.first] -= b;
                it = P.free.erase(it);
            } else {
                ++it;
            }
        }
    }
    for (void* q : drop) cudaFree(q);
    return drop.size();
}

// Idle bytes the pool keeps per device: a quarter of its memory, so a long
// run of contexts of changing sizes cannot park the whole device in the cache.
size_t pool_cap(int device) {
    DevicePool& P = pool();
    auto it = P.cap.find(device);
    if (it != P.cap.end()) return it->second;
    cudaDeviceProp prop;
    const size_t c = cudaGetDeviceProperties(&prop, device) == cudaSuccess ? prop.totalGlobalMem / 4 : (size_t)8 << 30;
    P.cap[device] = c;
    return c;
}

cudaError_t pool_alloc(int device, void** p, size_t bytes) {
    DevicePool& P = pool();
    const size_t cls = size_class(bytes);
    {
        std::lock_guard<std::mutex> g(P.m);
        auto it = P.free.find({device, cls});
        if (it != P.free.end() && !it->second.empty()) {
            *p = it->second.back();
            it->second.pop_back();
            P.cached -= cls;
            P.cached_on[device] -= cls;
            P.live[*p] = {device, cls};
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMalloc(p, cls);
    for (int attempt = 0; e != cudaSuccess && attempt < 2; attempt++) {
        cudaGetLastError();
        pool_trim_device(device);
        e = cudaMalloc(p, cls);
    }
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> g(P.m);
        P.live[*p] = {device, cls};
    }
    return e;
}

void pool_free(void* p) {
    if (!p) return;
    DevicePool& P = pool();
    {
        std::lock_guard<std::mutex> g(P.m);
        auto it = P.live.find(p);
        if (it != P.live.end()) {
            const int dev = it->second.first;
            const size_t cls = it->second.second;
            if (P.cached_on[dev] + cls <= pool_cap(dev)) {
                P.free[it->second].push_back(p);
                P.cached += cls;
                P.cached_on[dev] += cls;
                P.live.erase(it);
                return;
            }
            P.live.erase(it);      // over the cap: released at once
        }
    }
    cudaFree(p);
}

template <class T>
int dalloc(hfem_ctx* c, T** p, size_t count) {
    if (*p) {
        cudaStreamSynchronize(c->stream);          // the old block may still be read by queued work
        pool_free(*p);
        *p = nullptr;
    }
    if (count == 0) count = 1;
    cudaError_t e = pool_alloc(c->device, (void**)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, HFEM_E_NOMEM, "device allocation of %zu bytes: %s", sizeof(T) * count, cudaGetErrorString(e));
    }
    return 0;
}

template <class T>
int upload(hfem_ctx* c, T** p, const T* h, size_t count) {
    int rc = dalloc(c, p, count);
    if (rc) return rc;
    CK(cudaMemcpyAsync(*p, h, sizeof(T) * count, cudaMemcpyHostToDevice, c->stream));
    return 0;
}

struct Timed {
    hfem_ctx* c;
    const char* name;
    cudaEvent_t a = nullptr, b = nullptr;
    Timed(hfem_ctx* c_, const char* n) : c(c_), name(n) {
        if (c->timer.on) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, c->stream);
        }
    }
    ~Timed() {
        if (c->timer.on) {
            cudaEventRecord(b, c->stream);
            c->timer.pending.push_back({name, {a, b}});
        }
    }
};

void flush_timer(hfem_ctx* c) {
    for (auto& p : c->timer.pending) {
        cudaEventSynchronize(p.second.second);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.second.first, p.second.second);
        auto& slot = c->timer.acc[p.first];
        slot.first += ms;
        slot.second += 1;
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    c->timer.pending.clear();
}

int check_launch(hfem_ctx* c, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, HFEM_E_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
    return 0;
}

int sms(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v > 0 ? v : 1;
}

int ensure_assembly_buffers(hfem_ctx* c) {
    if (c->D) return 0;
    const size_t ne = c->dims.ne, n = c->n, nb = c->nb;
    int rc = 0;
    if ((rc = dalloc(c, &c->D, ne * n * n))) return rc;
    if ((rc = dalloc(c, &c->F, ne * n * nb))) return rc;
    if ((rc = dalloc(c, &c->DinvF, ne * n * nb))) return rc;
    if ((rc = dalloc(c, &c->K, ne * nb * n))) return rc;
    if ((rc = dalloc(c, &c->H, ne * nb * nb))) return rc;
    if ((rc = dalloc(c, &c->Ru, ne * n))) return rc;
    if ((rc = dalloc(c, &c->DinvRu, ne * n))) return rc;
    if ((rc = dalloc(c, &c->Rh, ne * nb))) return rc;
    if ((rc = dalloc(c, &c->Ro, ne * nb))) return rc;
    if ((rc = dalloc(c, &c->ru2, ne))) return rc;
    if ((rc = dalloc(c, &c->info, ne))) return rc;
    if ((rc = dalloc(c, &c->ws, (size_t)c->grid_elem * c->L->ws))) return rc;
    if ((rc = dalloc(c, &c->tc_err, 1))) return rc;
    if ((rc = dalloc(c, &c->rn_part, RNORM_CTAS))) return rc;
    CK(cudaMemsetAsync(c->tc_err, 0, sizeof(int), c->stream));
    return 0;
}

ElemArgs elem_args(hfem_ctx* c) {
    ElemArgs a;
    a.inviscid = c->appname == 0;
    a.conv_stab = c->conv_stab;
    a.visc_model = c->visc_model;
    a.err = c->tc_err;
    a.bf = c->bf;
    a.bcm = c->bcm;
    a.bcs = c->bcs;
    a.T = Tables{c->shapvt, c->shapvg, c->svsv, c->shapft, c->shapfg, c->sfsf, c->perm};
    a.dgnodes = c->dgnodes;
    a.elcon = c->elcon;
    a.udg = c->udg;
    a.uh = c->uh;
    a.sh = c->sh;
    for (int i = 0; i < 6; i++) a.param[i] = c->param[i];
    a.tdep = c->tdep;
    a.fc_u = c->fc_u;
    a.fc_q = c->fc_q;
    a.ne = c->dims.ne;
    a.D = c->D; a.F = c->F; a.K = c->K; a.H = c->H;
    a.Ru = c->Ru; a.Rh = c->Rh; a.Ro = c->Ro; a.ru2 = c->ru2;
    a.ws = c->ws;
    a.eprob = c->nprob ? c->eprob : nullptr;
    a.pparam = c->nprob ? c->pparam : nullptr;
    return a;
}

ScatterArgs scatter_args(hfem_ctx* c) {
    ScatterArgs s;
    s.nblk = c->dims.nblocks; s.nf = c->dims.nf; s.npf = c->dims.npf; s.nch = c->nch; s.nfe = c->dims.nfe; s.nb = c->nb;
    s.blk_src = c->blk_src; s.face_src = c->face_src; s.elcon = c->elcon;
    s.rowface = c->rowface; s.colface = c->colface;
    s.H = c->H; s.Rh = c->Rh; s.Ro = c->Ro;
    s.Hg = c->Hg; s.Rg = c->Rg; s.Rr = c->Rr;
    return s;
}

// The interior-face lift D += P K (src = K, n columns) or F += P H (src = H,
// nb columns) applied by the condensation kernels (lift.cuh).
LiftArgs lift_args(hfem_ctx* c, const double* src, int cols) {
    LiftArgs L;
    L.src = src;
    L.perm = c->perm;
    L.bf = c->bf;
    L.npv = c->dims.npv;
    L.npf = c->dims.npf;
    L.nfe = c->dims.nfe;
    L.nch = c->nch;
    L.cols = cols;
    return L;
}

// F += P H (interior faces) in place, ahead of the condensation kernels.
int lift_F(hfem_ctx* c) {
    Timed t(c, "lift_F");
    const long long cols = (long long)c->dims.ne * c->nb;
    const int grid = (int)std::max(1LL, std::min(cols / LIFT_WARPS, (long long)sms(c->device) * 8));
    lift_inplace_kernel<<<grid, 32 * LIFT_WARPS, 0, c->stream>>>(c->dims.ne, c->n, lift_args(c, c->H, c->nb), c->F);
    return check_launch(c, "lift_F");
}

int ready(hfem_ctx* c) {
    if (!c) return HFEM_E_ARG;
    if (!c->have_master || !c->have_mesh || !c->have_phys || !c->have_sol)
        return fail(c, HFEM_E_STATE, "master, mesh, physics and solution must be set first");
    return 0;
}

// Element pass: local blocks, condensation (matrix=true) and scatter, as
// launches on the context's stream only (no host synchronisation, so the
// sequence can be captured into a CUDA graph).  Buffers must exist.
int enqueue_assembly(hfem_ctx* c, bool matrix) {
    int rc;
    const int tf = (c->precision == 1 || c->precision == 3) ? 1 : 0;
    const int gen = (c->conv_stab != 0 || c->visc_model != 0) ? 1 : 0;
    const dim3 ge(c->grid_elem_v[tf][gen]);
    auto element = c->L->element_v[tf][gen];
    {
        Timed t(c, "element");
        if (c->pending_chunks > 0) {
            // one launch per piece of the state, each after that piece's copy
            for (int k = 0; k < c->pending_chunks; k++) {
                CK(cudaStreamWaitEvent(c->stream, c->chunk_ev[k + 1], 0));
                ElemArgs a = elem_args(c);
                a.e_begin = c->chunk_lo[k];
                a.ne = c->chunk_lo[k + 1];
                element(ge, c->L->elem_smem, c->stream, a);
                if ((rc = check_launch(c, "element"))) return rc;
            }
            c->pending_chunks = 0;
        } else {
            element(ge, c->L->elem_smem, c->stream, elem_args(c));
            if ((rc = check_launch(c, "element"))) return rc;
        }
    }
    ScatterArgs sa = scatter_args(c);
    if (matrix) {
        const int ne = c->dims.ne, n = c->n, nb = c->nb;
        {
            Timed t(c, "inverse");
            // D^-1 Ru to its own buffer: residual-only passes (a Newton line
            // search) overwrite Ru while the update still needs D^-1 Ru
            c->L->inverse(dim3(c->grid_inv), c->stream, ne, c->D, c->Ru, c->DinvRu, c->info);
            if ((rc = check_launch(c, "inverse"))) return rc;
        }
        if (c->precision != 1 && c->g1_sel < 0 && c->g2_sel < 0) {
            // both products in one kernel (tilings chosen by hfem_set_gemm_tiles
            // or hfem_autotune run the two batched GEMMs instead)
            if ((rc = lift_F(c))) return rc;
            Timed t(c, "schur_fused");
            c->L->schur_fused(c->stream, ne, c->D, c->F, c->K, c->H, c->DinvF);
            if ((rc = check_launch(c, "schur_fused"))) return rc;
        } else if (c->precision != 1) {
            const GemmLaunch& g1 = c->g1_sel >= 0 ? gemm_candidates()[c->g1_sel] : c->L->g1;
            const GemmLaunch& g2 = c->g2_sel >= 0 ? gemm_candidates()[c->g2_sel] : c->L->g2;
            if ((rc = lift_F(c))) return rc;
            {
                Timed t(c, "gemm_DinvF");
                g1.run(c->stream, ne, n, nb, n, 1.0, c->D, n, (long long)n * n, c->F, n, (long long)n * nb, 0.0,
                       c->DinvF, n, (long long)n * nb);
                if ((rc = check_launch(c, "gemm_DinvF"))) return rc;
            }
            {
                Timed t(c, "gemm_schur");
                g2.run(c->stream, ne, nb, nb, n, -1.0, c->K, nb, (long long)nb * n, c->DinvF, n, (long long)n * nb,
                       1.0, c->H, nb, (long long)nb * nb);
                if ((rc = check_launch(c, "gemm_schur"))) return rc;
            }
        } else {
            if ((rc = lift_F(c))) return rc;
            Timed t(c, "schur_tc");
            SchurTcArgs ta{ne, c->D, c->F, c->K, c->H, c->DinvF, c->tc_err};
            c->L->schur_tc(dim3(c->grid_tc), c->L->tc_smem, c->stream, ta);
            if ((rc = check_launch(c, "schur_tc"))) return rc;
        }
        {
            Timed t(c, "gemv_Rh");
            batched_dgemv_kernel<<<sms(c->device) * 8, 256, 0, c->stream>>>(ne, nb, n, -1.0, c->K, (long long)nb * n,
                                                                           c->DinvRu, n, c->Rh, nb);
            if ((rc = check_launch(c, "gemv_Rh"))) return rc;
        }
        {
            Timed t(c, "scatter_H");
            c->L->scatter_h(dim3(std::max(1, std::min((c->dims.nblocks + 7) / 8, sms(c->device) * 8))), c->stream, sa);
            if ((rc = check_launch(c, "scatter_H"))) return rc;
        }
    } else {
        sa.Rg = nullptr;
    }
    {
        Timed t(c, "scatter_R");
        scatter_R_kernel<<<sms(c->device) * 4, 256, 0, c->stream>>>(sa);
        if ((rc = check_launch(c, "scatter_R"))) return rc;
    }
    rnorm_partial_kernel<<<RNORM_CTAS, 256, 0, c->stream>>>(c->dims.ne, c->ru2, (long long)c->dims.nf * c->bsz,
                                                            c->Rr, c->rn_part);
    rnorm_final_kernel<<<1, 32, 0, c->stream>>>(RNORM_CTAS, c->rn_part, c->rnorm);
    return check_launch(c, "rnorm");
}

// Wait for an enqueued assembly, check the element LUs (and the tensor-core
// kernel) and read the residual norm.
int finish_assembly(hfem_ctx* c, bool matrix, double* rnorm_out) {
    if (matrix) {
        std::vector<int> info(c->dims.ne);
        CK(cudaMemcpyAsync(info.data(), c->info, sizeof(int) * info.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int e = 0; e < c->dims.ne; e++)
            if (info[e]) return fail(c, HFEM_E_SINGULAR, "element %d: singular local matrix (pivot %d)", e, info[e]);
    }
    int terr = 0;
    CK(cudaMemcpyAsync(&terr, c->tc_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (terr == 1) return fail(c, HFEM_E_CUDA, "tensor-core Schur kernel: an MMA completion wait expired");
    if (terr == 2) return fail(c, HFEM_E_CUDA, "element kernel: a bulk-copy completion wait expired");
    if (matrix) c->assembled = true;
    double rn = 0.0;
    CK(cudaMemcpyAsync(&rn, c->rnorm, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    flush_timer(c);
    if (rnorm_out) *rnorm_out = rn;
    return 0;
}

int run_assembly(hfem_ctx* c, bool matrix, double* rnorm_out) {
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = ensure_assembly_buffers(c))) return rc;
    if ((rc = enqueue_assembly(c, matrix))) return rc;
    return finish_assembly(c, matrix, rnorm_out);
}

int launch_getq(hfem_ctx* c, const double* duh, double alpha) {
    QArgs q;
    q.T = Tables{c->shapvt, c->shapvg, c->svsv, c->shapft, c->shapfg, c->sfsf, c->perm};
    q.dgnodes = c->dgnodes;
    q.elcon = c->elcon;
    q.udg = c->udg;
    q.uh = c->uh;
    q.sh = c->sh;
    q.fc_q = c->fc_q;
    q.ne = c->dims.ne;
    q.DinvRu = duh ? c->DinvRu : nullptr;
    q.DinvF = duh ? c->DinvF : nullptr;
    q.duh = duh;
    q.alpha = alpha;
    q.eprob = c->eprob;
    q.palpha = (duh && c->nprob && c->palpha_on) ? c->palpha : nullptr;
    Timed t(c, duh ? "update" : "getq");
    c->L->getq(dim3(c->grid_elem), c->L->q_smem, c->stream, q);
    return check_launch(c, "getq");
}

long long nvec(hfem_ctx* c) { return (long long)c->dims.nf * c->bsz; }

int dot(hfem_ctx* c, const double* a, const double* b, double* out, bool sq) {
    dot_partial_kernel<<<DOT_CTAS, DOT_THREADS, 0, c->stream>>>(nvec(c), a, b, c->part);
    dot_final_kernel<<<1, 256, 0, c->stream>>>(c->part, out, sq ? 1 : 0);
    return check_launch(c, "dot");
}

// ---------------------------------------------------------------- BILU0
// Block sizes with one-CTA (scheduled) instances of the factorisation and the
// solves; they run when the levels are short (few rows per level, as the MDF
// order gives), where a launch or a CTA per row of a level would leave the GPU
// waiting on the dependency chain.
bool bilu_sched_bsz(int b) { return b == 8 || b == 12 || b == 15 || b == 16 || b == 20 || b == 30; }

// Same arithmetic as the LU of the oracle's restatement, so that the weights,
// and with them the ordering, are reproduced bit for bit.
int host_lu_factor(int n, double* a, int* piv) {
    for (int j = 0; j < n; j++) {
        int p = j;
        double m = std::fabs(a[j + n * j]);
        for (int i = j + 1; i < n; i++)
            if (std::fabs(a[i + n * j]) > m) { m = std::fabs(a[i + n * j]); p = i; }
        piv[j] = p;
        if (a[p + n * j] == 0.0) return j + 1;
        if (p != j) for (int k = 0; k < n; k++) std::swap(a[j + n * k], a[p + n * k]);
        const double inv = 1.0 / a[j + n * j];
        for (int i = j + 1; i < n; i++) a[i + n * j] *= inv;
        for (int k = j + 1; k < n; k++) {
            const double t = a[j + n * k];
            if (t != 0.0) for (int i = j + 1; i < n; i++) a[i + n * k] -= a[i + n * j] * t;
        }
    }
    return 0;
}
void host_lu_solve(int n, const double* lu, const int* piv, int nrhs, double* b) {
    for (int r = 0; r < nrhs; r++) {
        double* x = b + (size_t)n * r;
        for (int i = 0; i < n; i++) if (piv[i] != i) std::swap(x[i], x[piv[i]]);
        for (int i = 0; i < n; i++) { double t = x[i]; for (int k = 0; k < i; k++) t -= lu[i + n * k] * x[k]; x[i] = t; }
        for (int i = n - 1; i >= 0; i--) {
            double t = x[i];
            for (int k = i + 1; k < n; k++) t -= lu[i + n * k] * x[k];
            x[i] = t / lu[i + n * i];
        }
    }
}

int row_find(const std::vector<int>& rs, const std::vector<int>& ci, int r, int col) {
    for (int k = rs[r]; k < rs[r + 1]; k++)
        if (ci[k] == col) return k;
    return -1;
}

// Minimum discarded fill ordering (kernel/computeMDFordering.m:1-150) of the
// current Hg, with a lazy min-heap keyed (weight, row) in place of the
// reference's linear search for the first minimum -- the same choice at every
// step -- and the level schedule of the factorisation and of both solves.
int compute_ordering(hfem_ctx* c) {
    const int nf = c->dims.nf, b = c->bsz;
    const size_t b2 = (size_t)b * b;
    const std::vector<int>& rs = c->h_rowstart;
    const std::vector<int>& ci = c->h_colidx;
    const int nblk = rs[nf];
    std::vector<double> Hg(b2 * nblk);
    CK(cudaMemcpyAsync(Hg.data(), c->Hg, sizeof(double) * Hg.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<double> C(nblk), a(b2), t(b2);
    std::vector<int> piv(b);
    for (int i = 0; i < nf; i++) {
        std::memcpy(a.data(), &Hg[b2 * rs[i]], sizeof(double) * b2);
        if (host_lu_factor(b, a.data(), piv.data())) return fail(c, HFEM_E_SINGULAR, "diagonal block of face %d", i);
        for (int n = rs[i]; n < rs[i + 1]; n++) {
            std::memcpy(t.data(), &Hg[b2 * n], sizeof(double) * b2);
            host_lu_solve(b, a.data(), piv.data(), b, t.data());
            double s = 0.0;
            for (size_t q = 0; q < b2; q++) s += t[q] * t[q];
            C[n] = std::sqrt(s);
        }
    }
    const double big = 1e100;
    std::vector<double> w(nf);
    std::vector<int> pos;
    auto weight = [&](int k) {
        double s = 0.0;
        for (size_t ii = 0; ii < pos.size(); ii++) {
            const int ri = ci[pos[ii]];
            const double Cik = C[row_find(rs, ci, ri, k)];
            for (size_t jj = 0; jj < pos.size(); jj++) {
                if (jj == ii) continue;
                if (row_find(rs, ci, ri, ci[pos[jj]]) < 0) {
                    const double v = Cik * C[pos[jj]];
                    s += v * v;
                }
            }
        }
        return std::sqrt(s);
    };
    using Item = std::pair<double, int>;
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
    for (int k = 0; k < nf; k++) {
        pos.clear();
        for (int q = rs[k] + 1; q < rs[k + 1]; q++) pos.push_back(q);
        w[k] = weight(k);
        heap.push({w[k], k});
    }
    c->h_o2u.assign(nf, 0);
    c->h_u2o.assign(nf, 0);
    for (int l = 0; l < nf; l++) {
        int p = -1;
        while (!heap.empty()) {
            const Item it = heap.top();
            heap.pop();
            if (w[it.second] < big && it.first == w[it.second]) { p = it.second; break; }
        }
        if (p < 0) return fail(c, HFEM_E_STATE, "ordering heap exhausted");
        c->h_o2u[l] = p;
        w[p] = big;
        for (int e = rs[p] + 1; e < rs[p + 1]; e++) {
            const int k = ci[e];
            if (!(w[k] < big)) continue;
            pos.clear();
            for (int q = rs[k] + 1; q < rs[k + 1]; q++)
                if (w[ci[q]] < big) pos.push_back(q);
            w[k] = weight(k);
            heap.push({w[k], k});
        }
    }
    for (int i = 0; i < nf; i++) c->h_u2o[c->h_o2u[i]] = i;
    // level schedule: lower (and factorisation) over earlier neighbours, upper over later ones
    const std::vector<int>& o2u = c->h_o2u;
    const std::vector<int>& u2o = c->h_u2o;
    std::vector<int> lev(nf, 0), levu(nf, 0);
    int nl = 0, nu = 0;
    for (int l = 0; l < nf; l++) {
        const int i = o2u[l];
        int m = 0;
        for (int q = rs[i] + 1; q < rs[i + 1]; q++)
            if (u2o[ci[q]] < l) m = std::max(m, lev[ci[q]] + 1);
        lev[i] = m;
        nl = std::max(nl, m + 1);
    }
    for (int l = nf - 1; l >= 0; l--) {
        const int i = o2u[l];
        int m = 0;
        for (int q = rs[i] + 1; q < rs[i + 1]; q++)
            if (u2o[ci[q]] > l) m = std::max(m, levu[ci[q]] + 1);
        levu[i] = m;
        nu = std::max(nu, m + 1);
    }
    auto group = [&](const std::vector<int>& L, int nlev, std::vector<int>& ptr) {
        ptr.assign(nlev + 1, 0);
        for (int i = 0; i < nf; i++) ptr[L[i] + 1]++;
        for (int k = 0; k < nlev; k++) ptr[k + 1] += ptr[k];
        std::vector<int> rows(nf), fill(ptr.begin(), ptr.end() - 1);
        for (int l = 0; l < nf; l++) rows[fill[L[o2u[l]]]++] = o2u[l];
        return rows;
    };
    const std::vector<int> rows_lo = group(lev, nl, c->lvl_lo);
    const std::vector<int> rows_up = group(levu, nu, c->lvl_up);
    // per row, the positions of its earlier neighbours in increasing order
    std::vector<int> fptr(nf + 1, 0), fpos;
    for (int i = 0; i < nf; i++) {
        std::vector<std::pair<int, int>> e;
        for (int q = rs[i] + 1; q < rs[i + 1]; q++)
            if (u2o[ci[q]] < u2o[i]) e.push_back({u2o[ci[q]], q});
        std::sort(e.begin(), e.end());
        for (auto& x : e) fpos.push_back(x.second);
        fptr[i + 1] = (int)fpos.size();
    }
    if (fpos.empty()) fpos.push_back(0);
    // a new ordering (hfem_reset_ordering) replaces the previous one's tables
    for (int** q : {&c->d_u2o, &c->d_rows_lo, &c->d_rows_up, &c->d_fptr, &c->d_fpos, &c->d_lvl_lo, &c->d_lvl_up,
                    &c->d_frec, &c->d_lrec, &c->d_urec})
        if (*q) {
            pool_free(*q);
            *q = nullptr;
        }
    // per-slot records of the one-CTA forms (BiluSched), when the block size
    // has an instance, the levels are short and every row fits their limits
    std::vector<int> frec, lrec, urec;
    c->bilu_sched = bilu_sched_bsz(b) && (long long)nf < 32LL * std::max(nl, nu);
    for (int s = 0; s < nf && c->bilu_sched; s++) {
        const int i = rows_lo[s];
        if (rs[i + 1] - rs[i] > BILU_ROWMAX) c->bilu_sched = false;
    }
    if (c->bilu_sched) {
        frec.assign((size_t)nf * BILU_FREC, 0);
        lrec.assign((size_t)nf * BILU_SREC, 0);
        urec.assign((size_t)nf * BILU_SREC, 0);
        for (int s = 0; s < nf && c->bilu_sched; s++) {
            const int i = rows_lo[s];
            int* F = &frec[(size_t)s * BILU_FREC];
            F[0] = i;
            F[1] = rs[i];
            F[2] = rs[i + 1] - rs[i];
            int nr = 0, nuu = 0;
            for (int f = fptr[i]; f < fptr[i + 1] && c->bilu_sched; f++) {
                const int p = fpos[f], k = ci[p];
                if (nr >= 32 || nuu >= 32) { c->bilu_sched = false; break; }
                const int head = nr++;
                F[8 + 2 * head] = p - rs[i];
                F[72 + nuu++] = rs[k];
                for (int q = rs[i]; q < rs[i + 1]; q++) {
                    const int l = ci[q];
                    if (u2o[l] <= u2o[k]) continue;
                    const int m = row_find(rs, ci, k, l);
                    if (m < 0) continue;
                    if (nr >= 32 || nuu >= 32) { c->bilu_sched = false; break; }
                    F[8 + 2 * nr++] = q - rs[i];
                    F[72 + nuu++] = m;
                    F[9 + 2 * head]++;
                }
            }
            F[3] = nr;
            F[4] = nuu;
            int* L = &lrec[(size_t)s * BILU_SREC];
            L[0] = i;
            for (int q = rs[i] + 1; q < rs[i + 1]; q++)
                if (u2o[ci[q]] < u2o[i]) {
                    L[4 + 2 * L[1]] = q;
                    L[5 + 2 * L[1]] = ci[q];
                    L[1]++;
                }
        }
        for (int s = 0; s < nf; s++) {
            const int i = rows_up[s];
            int* U = &urec[(size_t)s * BILU_SREC];
            U[0] = i;
            U[2] = rs[i];
            for (int q = rs[i] + 1; q < rs[i + 1]; q++)
                if (u2o[ci[q]] > u2o[i]) {
                    U[4 + 2 * U[1]] = q;
                    U[5 + 2 * U[1]] = ci[q];
                    U[1]++;
                }
        }
        // slots: row i's result is live from its level to the last level that
        // reads it (later neighbours in the lower solve, earlier ones in the
        // upper); rows take the free slots of ranges that ended before their level
        auto assign = [&](const std::vector<int>& L, const std::vector<int>& ptr, const std::vector<int>& rows,
                          bool lower, std::vector<int>& rec) {
            const int nlev = (int)ptr.size() - 1;
            std::vector<int> end(L), slot(nf, 0), freed_ptr(nlev + 1, 0), freed(nf), free_list;
            for (int i = 0; i < nf; i++)
                for (int q = rs[i] + 1; q < rs[i + 1]; q++) {
                    const int k = ci[q];
                    if (lower ? u2o[k] > u2o[i] : u2o[k] < u2o[i]) end[i] = std::max(end[i], L[k]);
                }
            for (int i = 0; i < nf; i++) freed_ptr[end[i] + 1]++;
            for (int l = 0; l < nlev; l++) freed_ptr[l + 1] += freed_ptr[l];
            {
                std::vector<int> fill(freed_ptr.begin(), freed_ptr.end() - 1);
                for (int i = 0; i < nf; i++) freed[fill[end[i]]++] = i;
            }
            int n = 0;
            for (int l = 0; l < nlev; l++) {
                if (l > 0)
                    for (int t = freed_ptr[l - 1]; t < freed_ptr[l]; t++) free_list.push_back(slot[freed[t]]);
                for (int t = ptr[l]; t < ptr[l + 1]; t++) {
                    const int i = rows[t];
                    if (free_list.empty()) slot[i] = n++;
                    else {
                        slot[i] = free_list.back();
                        free_list.pop_back();
                    }
                }
            }
            for (int t = 0; t < nf; t++) {
                int* R = &rec[(size_t)t * BILU_SREC];
                R[3] = slot[R[0]];
                for (int j = 0; j < R[1]; j++) R[16 + j] = slot[R[5 + 2 * j]];
            }
            return n;
        };
        c->bilu_nslot_lo = assign(lev, c->lvl_lo, rows_lo, true, lrec);
        c->bilu_nslot_up = assign(levu, c->lvl_up, rows_up, false, urec);
    }
    int rc;
    if ((rc = upload(c, &c->d_u2o, u2o.data(), (size_t)nf)) || (rc = upload(c, &c->d_rows_lo, rows_lo.data(), (size_t)nf)) ||
        (rc = upload(c, &c->d_rows_up, rows_up.data(), (size_t)nf)) ||
        (rc = upload(c, &c->d_fptr, fptr.data(), fptr.size())) || (rc = upload(c, &c->d_fpos, fpos.data(), fpos.size())) ||
        (rc = upload(c, &c->d_lvl_lo, c->lvl_lo.data(), c->lvl_lo.size())) ||
        (rc = upload(c, &c->d_lvl_up, c->lvl_up.data(), c->lvl_up.size())) ||
        (c->bilu_sched && ((rc = upload(c, &c->d_frec, frec.data(), frec.size())) ||
                           (rc = upload(c, &c->d_lrec, lrec.data(), lrec.size())) ||
                           (rc = upload(c, &c->d_urec, urec.data(), urec.size())))))
        return rc;
    if (!c->Mg && (rc = dalloc(c, &c->Mg, b2 * nblk))) return rc;
    if (!c->bl_t && (rc = dalloc(c, &c->bl_t, (size_t)nf * b))) return rc;
    if (!c->bl_y && (rc = dalloc(c, &c->bl_y, (size_t)nf * b))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    if (c->bilu_exec) {
        cudaGraphExecDestroy(c->bilu_exec);
        c->bilu_exec = nullptr;
    }
    c->have_order = true;
    return 0;
}

BiluSched bilu_sched_args(const hfem_ctx* c) {
    return BiluSched{(int)c->lvl_lo.size() - 1, (int)c->lvl_up.size() - 1, c->d_lvl_lo, c->d_lvl_up,
                     c->d_frec, c->d_lrec, c->d_urec, c->bilu_nslot_lo, c->bilu_nslot_up};
}

template <int B>
void launch_bilu_factor_sched(hfem_ctx* c, const BiluSched& S) {
    using C = BiluFacCfg<B>;
    cudaFuncSetAttribute(bilu0_factor_sched_kernel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    bilu0_factor_sched_kernel<B><<<1, 32 * C::NW, C::SMEM, c->stream>>>(S, c->Mg, c->binfo);
}
template <int B, class MT>
void launch_bilu_solve_sched(hfem_ctx* c, BiluSched S, const MT* M, const double* x, double* v) {
    using C = BiluSolCfg<B, MT>;
    int nslot = std::max(S.nslot_lo, S.nslot_up), nw = C::warps(nslot);
    if (nw == 0) {   // results too many to keep: read them from global memory
        S.nslot_lo = S.nslot_up = nslot = 0;
        nw = C::warps(0);
    }
    const size_t smem = C::smem(nw, nslot);
    cudaFuncSetAttribute(bilu0_solve_sched_kernel<B, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    bilu0_solve_sched_kernel<B, MT><<<1, 32 * nw, smem, c->stream>>>(S, M, x, c->bl_y, v);
}

void enqueue_bilu0_levels(hfem_ctx* c, cudaStream_t st) {
    const int b = c->bsz;
    const size_t b2 = (size_t)b * b;
    BiluArgs a{b, c->rowstart, c->colidx, c->d_u2o, nullptr, 0, c->d_fptr, c->d_fpos, c->Mg, c->binfo};
    const size_t smem = sizeof(double) * (2 * b2 + b) + sizeof(int) * b;
    for (size_t l = 0; l + 1 < c->lvl_lo.size(); l++) {
        a.rows = c->d_rows_lo + c->lvl_lo[l];
        a.nrows = c->lvl_lo[l + 1] - c->lvl_lo[l];
        bilu0_factor_kernel<<<std::min(a.nrows, sms(c->device) * 8), BILU_THREADS, smem, st>>>(a);
    }
}

// Factor Hg into Mg level by level (computeBILU0.m).  The level launches are
// captured once per ordering (on a private stream) and replayed as a graph.
int bilu0_factor(hfem_ctx* c) {
    Timed t(c, "bilu0_factor");
    const int nf = c->dims.nf, b = c->bsz;
    const size_t b2 = (size_t)b * b;
    CK(cudaMemcpyAsync(c->Mg, c->Hg, sizeof(double) * b2 * c->dims.nblocks, cudaMemcpyDeviceToDevice, c->stream));
    if (c->bilu_sched) {
        const BiluSched S = bilu_sched_args(c);
        switch (b) {
#define HFEM_BF(B) \
    case B: launch_bilu_factor_sched<B>(c, S); break;
            HFEM_BF(8) HFEM_BF(12) HFEM_BF(15) HFEM_BF(16) HFEM_BF(20) HFEM_BF(30)
#undef HFEM_BF
            default: break;
        }
    } else if (!c->bilu_exec) {
        cudaStream_t cap = nullptr;
        cudaGraph_t g = nullptr;
        if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            enqueue_bilu0_levels(c, cap);
            if (cudaStreamEndCapture(cap, &g) == cudaSuccess && g) {
                if (cudaGraphInstantiate(&c->bilu_exec, g, 0) != cudaSuccess) c->bilu_exec = nullptr;
                cudaGraphDestroy(g);
            }
        }
        if (cap) cudaStreamDestroy(cap);
        cudaGetLastError();
    }
    if (c->bilu_sched) {
    } else if (c->bilu_exec) CK(cudaGraphLaunch(c->bilu_exec, c->stream));
    else enqueue_bilu0_levels(c, c->stream);
    int rc = check_launch(c, "bilu0_factor");
    if (rc) return rc;
    std::vector<int> bi(nf);
    CK(cudaMemcpyAsync(bi.data(), c->binfo, sizeof(int) * nf, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < nf; i++)
        if (bi[i]) return fail(c, HFEM_E_SINGULAR, "BILU0: singular pivot block at face %d", i);
    if (c->precision >= 1) {
        // mixed precision: the triangular solves read FP32 factors (FP64 vectors and sums)
        const long long nm = (long long)b2 * c->dims.nblocks;
        if (!c->Mg32 && (rc = dalloc(c, &c->Mg32, (size_t)nm))) return rc;
        to_float_kernel<<<sms(c->device) * 4, 256, 0, c->stream>>>(nm, c->Mg, c->Mg32);
        if ((rc = check_launch(c, "bilu0_factor fp32"))) return rc;
    }
    return 0;
}

// v = (L U)^-1 x (applyBILU0.m); v may not alias x.
int bilu0_apply(hfem_ctx* c, const double* x, double* v) {
    Timed t(c, "bilu0_apply");
    const bool f32 = c->precision >= 1 && c->Mg32;
    BiluSolveArgs a{c->bsz, c->rowstart, c->colidx, c->d_u2o, nullptr, 0, f32 ? (const void*)c->Mg32 : c->Mg, x,
                    c->bl_y, v};
    const int nlo = (int)c->lvl_lo.size() - 1, nup = (int)c->lvl_up.size() - 1;
    if (c->bilu_sched) {
        const BiluSched S = bilu_sched_args(c);
        switch (c->bsz) {
#define HFEM_BS(B)                                                          \
    case B:                                                                 \
        if (f32) launch_bilu_solve_sched<B, float>(c, S, c->Mg32, x, v);     \
        else launch_bilu_solve_sched<B, double>(c, S, c->Mg, x, v);          \
        break;
            HFEM_BS(8) HFEM_BS(12) HFEM_BS(15) HFEM_BS(16) HFEM_BS(20) HFEM_BS(30)
#undef HFEM_BS
            default: break;
        }
        return check_launch(c, "bilu0_apply");
    }
    // few rows per level: one CTA walks all levels (no launch per level)
    if ((long long)c->dims.nf < 64LL * std::max(nlo, nup)) {
        if (f32)
            bilu0_apply_cta_kernel<float><<<1, 1024, 0, c->stream>>>(a, c->d_lvl_lo, nlo, c->d_rows_lo, c->d_lvl_up,
                                                                     nup, c->d_rows_up);
        else
            bilu0_apply_cta_kernel<double><<<1, 1024, 0, c->stream>>>(a, c->d_lvl_lo, nlo, c->d_rows_lo, c->d_lvl_up,
                                                                      nup, c->d_rows_up);
        return check_launch(c, "bilu0_apply");
    }
    for (size_t l = 0; l + 1 < c->lvl_lo.size(); l++) {
        a.rows = c->d_rows_lo + c->lvl_lo[l];
        a.nrows = c->lvl_lo[l + 1] - c->lvl_lo[l];
        if (f32) bilu0_lower_kernel<float><<<std::min(a.nrows, sms(c->device) * 16), 64, 0, c->stream>>>(a);
        else bilu0_lower_kernel<double><<<std::min(a.nrows, sms(c->device) * 16), 64, 0, c->stream>>>(a);
    }
    for (size_t l = 0; l + 1 < c->lvl_up.size(); l++) {
        a.rows = c->d_rows_up + c->lvl_up[l];
        a.nrows = c->lvl_up[l + 1] - c->lvl_up[l];
        if (f32) bilu0_upper_kernel<float><<<std::min(a.nrows, sms(c->device) * 16), 64, 0, c->stream>>>(a);
        else bilu0_upper_kernel<double><<<std::min(a.nrows, sms(c->device) * 16), 64, 0, c->stream>>>(a);
    }
    return check_launch(c, "bilu0_apply");
}

int matvec_prec(hfem_ctx* c, const double* x, double* z, bool prec) {
    Timed t(c, "matvec");
    if (prec && c->prec_kind == 0) {
        bsr_matvec_bj_kernel<double><<<std::min(c->dims.nf, sms(c->device) * 16), 64, sizeof(double) * 64, c->stream>>>(
            c->dims.nf, c->bsz, c->rowstart, c->colidx, c->Hg, (const double*)nullptr, x, c->bl_t);
        int rc = check_launch(c, "matvec");
        if (rc) return rc;
        return bilu0_apply(c, c->bl_t, z);
    }
    if (prec && c->precision >= 1)
        bsr_matvec_bj_kernel<float><<<std::min(c->dims.nf, sms(c->device) * 16), 64, sizeof(double) * 64, c->stream>>>(
            c->dims.nf, c->bsz, c->rowstart, c->colidx, c->Hg, c->Minv32, x, z);
    else
        bsr_matvec_bj_kernel<double><<<std::min(c->dims.nf, sms(c->device) * 16), 64, sizeof(double) * 64, c->stream>>>(
            c->dims.nf, c->bsz, c->rowstart, c->colidx, c->Hg, prec ? c->Minv : nullptr, x, z);
    return check_launch(c, "matvec");
}

int ensure_krylov(hfem_ctx* c, int restart) {
    int rc;
    const size_t n = nvec(c);
    if (!c->x) {
        if ((rc = dalloc(c, &c->x, n))) return rc;
        if ((rc = dalloc(c, &c->w, n))) return rc;
        if ((rc = dalloc(c, &c->pb, n))) return rc;
        if ((rc = dalloc(c, &c->Minv, (size_t)c->dims.nf * c->bsz * c->bsz))) return rc;
        if ((rc = dalloc(c, &c->part, DOT_CTAS))) return rc;
        if ((rc = dalloc(c, &c->binfo, c->dims.nf))) return rc;
    }
    if (c->krylov_restart < restart) {
        if ((rc = dalloc(c, &c->V, n * (restart + 1)))) return rc;
        if ((rc = dalloc(c, &c->scal, (size_t)(restart + 2) * (restart + 2)))) return rc;
        c->krylov_restart = restart;
    }
    return 0;
}

// Diagonal block of every face row -> contiguous blocks (for the blocked inverse).
__global__ void gather_diag_kernel(int nrows, int b2, const int* __restrict__ rowstart, const double* __restrict__ Hg,
                                   double* __restrict__ out) {
    const long long tot = (long long)nrows * b2;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x)
        out[t] = Hg[(size_t)rowstart[t / b2] * b2 + t % b2];
}

template <int B>
int bj_blocked(hfem_ctx* c) {
    cudaFuncSetAttribute(inverse_blocked_kernel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)InvBlk<B>::SMEM);
    const int nf = c->dims.nf;
    gather_diag_kernel<<<sms(c->device) * 8, 256, 0, c->stream>>>(nf, B * B, c->rowstart, c->Hg, c->Minv);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, inverse_blocked_kernel<B>, InvBlk<B>::THREADS, InvBlk<B>::SMEM);
    const int grid = std::max(1, std::min(nf, sms(c->device) * std::max(occ, 1)));
    // the kernel also solves with a right-hand side: c->w is free here and its
    // result is ignored
    inverse_blocked_kernel<B><<<grid, InvBlk<B>::THREADS, InvBlk<B>::SMEM, c->stream>>>(nf, c->Minv, c->w, c->w,
                                                                                     c->binfo);
    return check_launch(c, "bj_inverse");
}

// Block-Jacobi factor: Minv_i = inv(Hg_ii) for every face row (binfo[i] = 1 +
// pivot step of a singular block).  Block sizes with a blocked Gauss-Jordan
// instance take it (diagonal blocks gathered first); the others the one-CTA-
// per-block kernel.
int bj_factor(hfem_ctx* c) {
    Timed t(c, "bj_inverse");
    switch (c->bsz) {
        case 12: return bj_blocked<12>(c);
        case 16: return bj_blocked<16>(c);
        case 20: return bj_blocked<20>(c);
        case 30: return bj_blocked<30>(c);
        case 50: return bj_blocked<50>(c);
        default: break;
    }
    const size_t smem = sizeof(double) * ((size_t)c->bsz * c->bsz + c->bsz) + sizeof(int) * c->bsz;
    bj_inverse_kernel<<<std::min(c->dims.nf, sms(c->device) * 8), 64, smem, c->stream>>>(
        c->dims.nf, c->bsz, c->rowstart, c->Hg, c->Minv, c->binfo);
    return check_launch(c, "bj_inverse");
}

int gmres_seg_impl(hfem_ctx* c, int precond, int restart, double tol, int maxit, int* conv, int* iters,
                   double* hist, int hist_len);

int gmres_impl(hfem_ctx* c, int precond, int restart, double tol, int maxit, int* conv, int* iters, double* hist,
               int hist_len) {
    // one problem, block Jacobi or none: the fused single-segment kernels
    if (c->nprob == 0 && precond != 0 && c->assembled)
        return gmres_seg_impl(c, precond, restart, tol, maxit, conv, iters, hist, hist_len);
    int rc;
    if (!c->assembled) return fail(c, HFEM_E_STATE, "assemble before gmres");
    if (restart < 1 || maxit < 1 || !(tol > 0.0)) return fail(c, HFEM_E_ARG, "restart, maxit and tol must be positive");
    if (precond != -1 && precond != 0 && precond != 2)
        return fail(c, HFEM_E_ARG, "precond must be -1 (none), 0 (BILU0) or 2 (block Jacobi)");
    if ((rc = ensure_krylov(c, restart))) return rc;
    const long long n = nvec(c);
    const int g = sms(c->device) * 4;
    const bool prec = precond != -1;
    c->prec_kind = precond;
    if (precond == 0) {
        if (!c->have_order && (rc = compute_ordering(c))) return rc;
        if ((rc = bilu0_factor(c))) return rc;
        if ((rc = bilu0_apply(c, c->Rg, c->pb))) return rc;
    } else if (prec) {
        if ((rc = bj_factor(c))) return rc;
        std::vector<int> bi(c->dims.nf);
        CK(cudaMemcpyAsync(bi.data(), c->binfo, sizeof(int) * bi.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < c->dims.nf; i++)
            if (bi[i]) return fail(c, HFEM_E_SINGULAR, "diagonal block of face %d is singular", i);
        if (c->precision >= 1) {
            const long long nm = (long long)c->dims.nf * c->bsz * c->bsz;
            if (!c->Minv32 && (rc = dalloc(c, &c->Minv32, (size_t)nm))) return rc;
            to_float_kernel<<<g, 256, 0, c->stream>>>(nm, c->Minv, c->Minv32);
            bj_apply_kernel<float><<<g, 256, 0, c->stream>>>(c->dims.nf, c->bsz, c->Minv32, c->Rg, c->pb);
        } else {
            bj_apply_kernel<double><<<g, 256, 0, c->stream>>>(c->dims.nf, c->bsz, c->Minv, c->Rg, c->pb);
        }
    } else {
        CK(cudaMemcpyAsync(c->pb, c->Rg, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    }
    CK(cudaMemsetAsync(c->x, 0, sizeof(double) * n, c->stream));
    // scal layout: [0] nrmb, [1] beta, [2 .. 2+restart] current Hessenberg column, [..] y
    double* d_nrmb = c->scal;
    double* d_beta = c->scal + 1;
    double* d_h = c->scal + 2;
    double* d_y = c->scal + 3 + restart;
    if ((rc = dot(c, c->pb, c->pb, d_nrmb, true))) return rc;
    double nrmb = 0.0;
    CK(cudaMemcpyAsync(&nrmb, d_nrmb, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (nrmb == 0.0) nrmb = 1.0;
    std::vector<double> h((size_t)(restart + 1) * restart), cs(restart), sn(restart), gv(restart + 1), y(restart),
        hcol(restart + 2);
    int it = 0, flag = -2;
    while (flag == -2) {
        // r = M^-1 (b - A x) computed as M^-1 b - M^-1 A x (the same left-preconditioned residual)
        if ((rc = matvec_prec(c, c->x, c->w, prec))) return rc;
        sub_from_kernel<<<g, 256, 0, c->stream>>>(n, c->pb, c->w);
        if ((rc = dot(c, c->w, c->w, d_beta, true))) return rc;
        double beta = 0.0;
        CK(cudaMemcpyAsync(&beta, d_beta, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (beta / nrmb <= tol) { flag = 0; break; }
        scale_dev_kernel<<<g, 256, 0, c->stream>>>(n, d_beta, c->w, c->V);
        std::fill(gv.begin(), gv.end(), 0.0);
        gv[0] = beta;
        int j = 0;
        for (; j < restart; j++) {
            double* vj = c->V + (size_t)j * n;
            double* vn = c->V + (size_t)(j + 1) * n;
            if ((rc = matvec_prec(c, vj, vn, prec))) return rc;
            {
                Timed t(c, "orthogonalise");
                for (int i = 0; i <= j; i++) {             // modified Gram-Schmidt
                    if ((rc = dot(c, c->V + (size_t)i * n, vn, d_h + i, false))) return rc;
                    axpy_dev_kernel<<<g, 256, 0, c->stream>>>(n, d_h + i, c->V + (size_t)i * n, vn);
                }
                if ((rc = dot(c, vn, vn, d_h + j + 1, true))) return rc;
                scale_dev_kernel<<<g, 256, 0, c->stream>>>(n, d_h + j + 1, vn, vn);
            }
            CK(cudaMemcpyAsync(hcol.data(), d_h, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, c->stream));
            CK(cudaStreamSynchronize(c->stream));
            for (int i = 0; i <= j + 1; i++) h[i + (restart + 1) * j] = hcol[i];
            const double nn = hcol[j + 1];
            for (int i = 0; i < j; i++) {
                const double a = h[i + (restart + 1) * j], b = h[i + 1 + (restart + 1) * j];
                h[i + (restart + 1) * j] = cs[i] * a + sn[i] * b;
                h[i + 1 + (restart + 1) * j] = -sn[i] * a + cs[i] * b;
            }
            const double a = h[j + (restart + 1) * j], b = h[j + 1 + (restart + 1) * j];
            const double rr = std::sqrt(a * a + b * b);
            cs[j] = a / rr;
            sn[j] = b / rr;
            h[j + (restart + 1) * j] = rr;
            h[j + 1 + (restart + 1) * j] = 0.0;
            gv[j + 1] = -sn[j] * gv[j];
            gv[j] = cs[j] * gv[j];
            const double res = std::fabs(gv[j + 1]);
            if (hist && it < hist_len) hist[it] = res / nrmb;
            it++;
            if (res / nrmb <= tol) { flag = 0; j++; break; }
            if (it >= maxit) { flag = 1; j++; break; }
            if (nn == 0.0) { flag = -1; j++; break; }
        }
        for (int i = j - 1; i >= 0; i--) {
            double s = gv[i];
            for (int k = i + 1; k < j; k++) s -= h[i + (restart + 1) * k] * y[k];
            y[i] = s / h[i + (restart + 1) * i];
        }
        CK(cudaMemcpyAsync(d_y, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, c->stream));
        combine_kernel<<<g, 256, 0, c->stream>>>(n, j, c->V, d_y, c->x);
        if ((rc = check_launch(c, "combine"))) return rc;
    }
    CK(cudaStreamSynchronize(c->stream));
    flush_timer(c);
    if (iters) *iters = it;
    if (conv) *conv = (flag == 0) ? 1 : (flag == 1 ? 0 : -1);
    return 0;
}

// z = M^-1 Hg x (M^-1 omitted when !prec) by the warp-per-row kernel, rows
// of problems with act[p] == 0 skipped.
int matvec_warp(hfem_ctx* c, const double* x, double* z, bool prec, const unsigned char* act) {
    Timed t(c, "matvec_warp");
    const int grid = std::max(1, std::min((c->dims.nf + 7) / 8, sms(c->device) * 8));
    const double* M = prec ? c->Minv : nullptr;
    const int* rseg = act ? c->fprob : nullptr;
    switch (c->bsz) {
#define HFEM_MV(B)                                                                                                \
    case B:                                                                                                       \
        if (prec && c->precision >= 1)                                                                            \
            bsr_matvec_warp_kernel<B, float><<<grid, 256, 0, c->stream>>>(c->dims.nf, c->rowstart, c->colidx,      \
                                                                            c->Hg, c->Minv32, x, z, rseg, act);   \
        else                                                                                                      \
            bsr_matvec_warp_kernel<B, double><<<grid, 256, 0, c->stream>>>(c->dims.nf, c->rowstart, c->colidx,     \
                                                                             c->Hg, M, x, z, rseg, act);          \
        break;
        HFEM_MV(8) HFEM_MV(12) HFEM_MV(15) HFEM_MV(16) HFEM_MV(20) HFEM_MV(30) HFEM_MV(50)
#undef HFEM_MV
        default: return fail(c, HFEM_E_UNSUPPORTED, "no block matvec for block size %d", c->bsz);
    }
    return check_launch(c, "matvec_warp");
}

// Restarted, left-preconditioned GMRES with modified Gram-Schmidt run for
// every problem of the context at once (kernel/gmres_bilu0.m:17-105 per
// problem).  Each problem has its own Krylov basis (its segment of the
// vectors), Hessenberg matrix, Givens rotations and stopping test, so it takes
// exactly the iterations it takes alone; the launches are shared, and a
// problem that has stopped is skipped by every kernel.
// Segment tables for one segment over the whole trace vector (GMRES of a
// context without a problem map runs on the same fused kernels).
int ensure_single_segment(hfem_ctx* c) {
    if (c->seg_single) return 0;
    const long long ntot = (long long)c->dims.nf * c->bsz;
    long long piece = 1024;
    while (piece < SEG_PIECE && piece * 4 * sms(c->device) < ntot) piece *= 2;
    std::vector<long long> pstart;
    std::vector<int> pseg;
    for (long long s = 0; s < ntot; s += piece) {
        pstart.push_back(s);
        pseg.push_back(0);
    }
    pstart.push_back(ntot);
    const int p0[2] = {0, (int)pseg.size()};
    int rc;
    if ((rc = upload(c, &c->seg_pstart, pstart.data(), pstart.size())) ||
        (rc = upload(c, &c->seg_pseg, pseg.data(), pseg.size())) || (rc = upload(c, &c->seg_p0, p0, 2)) ||
        (rc = dalloc(c, &c->seg_ticket, 1)) || (rc = dalloc(c, &c->seg_part, pseg.size())) ||
        (rc = dalloc(c, &c->seg_nrm, 2)) || (rc = dalloc(c, &c->seg_act, 1)) || (rc = dalloc(c, &c->seg_k, 1)))
        return rc;
    CK(cudaMemsetAsync(c->seg_ticket, 0, sizeof(int), c->stream));
    c->npieces = (int)pseg.size();
    c->seg_restart = 0;
    c->seg_single = true;
    return 0;
}

int gmres_seg_impl(hfem_ctx* c, int precond, int restart, double tol, int maxit, int* conv, int* iters,
                   double* hist = nullptr, int hist_len = 0) {
    int rc;
    if (!c->assembled) return fail(c, HFEM_E_STATE, "assemble before gmres");
    const bool single = c->nprob == 0;
    if (single && (rc = ensure_single_segment(c))) return rc;
    if (!single && (!c->npieces || c->seg_single))
        return fail(c, HFEM_E_STATE, "per-problem GMRES needs a problem map with each problem's faces contiguous");
    if (restart < 1 || maxit < 1 || !(tol > 0.0)) return fail(c, HFEM_E_ARG, "restart, maxit and tol must be positive");
    if (precond != -1 && precond != 2) return fail(c, HFEM_E_ARG, "precond must be -1 (none) or 2 (block Jacobi)");
    if ((rc = ensure_krylov(c, restart))) return rc;
    const int P = single ? 1 : c->nprob;
    const unsigned char* mv_act = single ? nullptr : c->seg_act;   // row -> problem map only with a problem map
    if (c->seg_restart < restart || c->seg_hP < P) {
        // Hessenberg column (restart + 2 rows) and the second projection of
        // CGS2 (restart + 1 rows), P problems each
        if ((rc = dalloc(c, &c->seg_h, (size_t)(2 * restart + 3) * P))) return rc;
        if ((rc = dalloc(c, &c->seg_y, (size_t)restart * P))) return rc;
        if ((rc = dalloc(c, &c->gm_H, (size_t)(restart + 1) * restart * P)) ||
            (rc = dalloc(c, &c->gm_cs, (size_t)restart * P)) || (rc = dalloc(c, &c->gm_sn, (size_t)restart * P)) ||
            (rc = dalloc(c, &c->gm_g, (size_t)(restart + 1) * P)) || (rc = dalloc(c, &c->gm_nrmb, (size_t)P)) ||
            (rc = dalloc(c, &c->gm_state, (size_t)P)) || (rc = dalloc(c, &c->gm_its, (size_t)P)) ||
            (rc = dalloc(c, &c->gm_jc, (size_t)P)))
            return rc;
        c->seg_restart = restart;
        c->seg_hP = P;
    }
    const long long n = nvec(c);
    const int g = sms(c->device) * 4;
    const bool prec = precond == 2;
    // classical Gram-Schmidt with one reorthogonalisation (CGS2): 5 launches per
    // Arnoldi step instead of j + 3 for modified Gram-Schmidt.  It wins while
    // the steps are launch-bound, for small systems (measured on B200: 2D p=2,
    // 37k unknowns, 9.1 -> 5.9 ms per 62 steps); for larger ones the fused MGS
    // steps, which move the same bytes with more memory parallelism, win (3D
    // p=3, 2.5M unknowns: 33 ms with MGS, 75 ms with CGS2 per 69 steps; batches
    // of 2D requests, 0.3-2M unknowns, were slower with CGS2 too).
    const bool cgs2 = restart + 1 <= 64 && n <= (1ll << 17);
    if (hist && hist_len > 0 && c->gm_hist_n < (size_t)hist_len) {
        if ((rc = dalloc(c, &c->gm_hist, (size_t)hist_len))) return rc;
        c->gm_hist_n = (size_t)hist_len;
    }
    if (cgs2 && c->seg_partk_n < (size_t)c->npieces * (restart + 1)) {
        if ((rc = dalloc(c, &c->seg_partk, (size_t)c->npieces * (restart + 1)))) return rc;
        c->seg_partk_n = (size_t)c->npieces * (restart + 1);
    }
    if (prec) {
        if ((rc = bj_factor(c))) return rc;
        std::vector<int> bi(c->dims.nf);
        CK(cudaMemcpyAsync(bi.data(), c->binfo, sizeof(int) * bi.size(), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < c->dims.nf; i++)
            if (bi[i]) return fail(c, HFEM_E_SINGULAR, "diagonal block of face %d is singular", i);
        if (c->precision >= 1) {
            const long long nm = (long long)c->dims.nf * c->bsz * c->bsz;
            if (!c->Minv32 && (rc = dalloc(c, &c->Minv32, (size_t)nm))) return rc;
            to_float_kernel<<<g, 256, 0, c->stream>>>(nm, c->Minv, c->Minv32);
            bj_apply_kernel<float><<<g, 256, 0, c->stream>>>(c->dims.nf, c->bsz, c->Minv32, c->Rg, c->pb);
        } else {
            bj_apply_kernel<double><<<g, 256, 0, c->stream>>>(c->dims.nf, c->bsz, c->Minv, c->Rg, c->pb);
        }
    } else {
        CK(cudaMemcpyAsync(c->pb, c->Rg, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    }
    CK(cudaMemsetAsync(c->x, 0, sizeof(double) * n, c->stream));
    const SegPieces SP{c->npieces, c->seg_pstart, c->seg_pseg, c->seg_p0, c->seg_ticket, c->seg_part, c->seg_act};
    const int np = c->npieces;
    double* d_h = c->seg_h;                   // Hessenberg column, entry (i, p) at i * P + p
    double* d_h2 = c->seg_h + (size_t)(restart + 2) * P;   // CGS2's second projection, same layout
    // the Givens rotations, residual estimates and stopping tests run on the
    // device (gm_* kernels, one thread per problem); the host reads the
    // problems' masks back only every GM_CHECK steps and at the start of a
    // cycle, so the Arnoldi steps are enqueued without a round trip each
    constexpr int GM_CHECK = 8;
    const GmState GS{P, restart, maxit, tol, c->gm_H, c->gm_cs, c->gm_sn, c->gm_g, c->gm_nrmb, c->gm_state,
                     c->gm_its, c->gm_jc, c->seg_act, (hist && hist_len > 0) ? c->gm_hist : nullptr,
                     (hist && hist_len > 0) ? hist_len : 0};
    const int gb = (P + 127) / 128;
    std::vector<unsigned char> act(P, 1);
    auto set_act = [&]() -> int {
        CK(cudaMemcpyAsync(c->seg_act, act.data(), P, cudaMemcpyHostToDevice, c->stream));
        return 0;
    };
    auto any_active = [&](bool& live) -> int {
        CK(cudaMemcpyAsync(act.data(), c->seg_act, P, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        live = false;
        for (int p = 0; p < P; p++) live = live || act[p];
        return 0;
    };
    auto axpy_dot = [&](const double* hprev, const double* vprev, double* w, const double* b, double* out, int sq) {
        seg_axpy_dot_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, hprev, vprev, w, b, out, sq);
    };
    if ((rc = set_act())) return rc;
    axpy_dot(nullptr, nullptr, c->pb, c->pb, c->seg_nrm, 1);
    gm_init_kernel<<<gb, 128, 0, c->stream>>>(GS, c->seg_nrm);
    while (true) {
        // r = M^-1 b - M^-1 A x, beta = |r| per problem, on the problems still running
        gm_running_kernel<<<gb, 128, 0, c->stream>>>(GS);
        if ((rc = matvec_warp(c, c->x, c->w, prec, mv_act))) return rc;
        seg_sub_from_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, c->pb, c->w);
        axpy_dot(nullptr, nullptr, c->w, c->w, c->seg_nrm, 1);
        gm_cycle_kernel<<<gb, 128, 0, c->stream>>>(GS, c->seg_nrm);
        bool live = false;
        if ((rc = any_active(live))) return rc;
        if (!live) break;
        seg_scale_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, c->seg_nrm, c->w, c->V);
        for (int j = 0; j < restart && live; j++) {
            double* vj = c->V + (size_t)j * n;
            double* vn = c->V + (size_t)(j + 1) * n;
            if ((rc = matvec_warp(c, vj, vn, prec, mv_act))) return rc;
            {
                Timed t(c, "orthogonalise_seg");
                if (cgs2) {
                    const int k = j + 1;
                    seg_multidot_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, n, k, P, c->V, vn, c->seg_partk, d_h);
                    seg_update_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, n, k, P, c->V, d_h, vn, nullptr);
                    seg_multidot_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, n, k, P, c->V, vn, c->seg_partk,
                                                                           d_h2);
                    seg_update_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, n, k, P, c->V, d_h2, vn,
                                                                         d_h + (size_t)(j + 1) * P);
                } else {
                    for (int i = 0; i <= j; i++)
                        axpy_dot(i ? d_h + (size_t)(i - 1) * P : nullptr, i ? c->V + (size_t)(i - 1) * n : nullptr,
                                 vn, c->V + (size_t)i * n, d_h + (size_t)i * P, 0);
                    axpy_dot(d_h + (size_t)j * P, vj, vn, vn, d_h + (size_t)(j + 1) * P, 1);
                }
                seg_scale_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, d_h + (size_t)(j + 1) * P, vn, vn);
            }
            gm_givens_kernel<<<gb, 128, 0, c->stream>>>(GS, j, d_h, cgs2 ? d_h2 : nullptr);
            if ((rc = check_launch(c, "arnoldi"))) return rc;
            if ((j + 1) % GM_CHECK == 0 && j + 1 < restart && (rc = any_active(live))) return rc;
        }
        // x += V y for every problem that took part in this cycle
        gm_solve_kernel<<<gb, 128, 0, c->stream>>>(GS, c->seg_y, c->seg_k);
        seg_combine_kernel<<<np, SEG_THREADS, 0, c->stream>>>(SP, n, c->seg_k, restart, c->V, c->seg_y, c->x);
        if ((rc = check_launch(c, "combine_seg"))) return rc;
    }
    std::vector<int> state(P), its(P);
    CK(cudaMemcpyAsync(state.data(), c->gm_state, sizeof(int) * P, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(its.data(), c->gm_its, sizeof(int) * P, cudaMemcpyDeviceToHost, c->stream));
    if (hist && hist_len > 0)
        CK(cudaMemcpyAsync(hist, c->gm_hist, sizeof(double) * hist_len, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    flush_timer(c);
    for (int p = 0; p < P; p++) {
        if (conv) conv[p] = state[p] == 1 ? 1 : (state[p] == 0 ? 0 : -1);
        if (iters) iters[p] = its[p];
    }
    return 0;
}

int update_impl(hfem_ctx* c, double alpha) {
    int rc;
    if (!c->assembled || !c->x) return fail(c, HFEM_E_STATE, "assemble and solve before update");
    axpy_kernel<<<sms(c->device) * 4, 256, 0, c->stream>>>(nvec(c), alpha, c->x, c->uh);
    if ((rc = check_launch(c, "uh update"))) return rc;
    if ((rc = launch_getq(c, c->x, alpha))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    flush_timer(c);
    return 0;
}

// DIRK(s, q) tableaus (solvers/DIRKcoeff.cpp:6-118 lists the same methods):
// d = A^-1 column-major (d[i + s*j]), t = stage times c_i.  The tableaus are the
// published ones: backward Euler, implicit midpoint, the 2-stage L-stable SDIRK
// (gamma = 1 - 1/sqrt 2), the 2-stage 3rd-order SDIRK (gamma = (3 + sqrt 3)/6) and
// Alexander's 3-stage L-stable SDIRK (gamma the root of g^3 - 3g^2 + 3g/2 - 1/6 in (0,1)).
bool dirk_table(int stages, int order, double* d, double* t) {
    double A[9] = {0};
    if (stages == 1 && order == 1) { A[0] = 1.0; t[0] = 1.0; }
    else if (stages == 1 && order == 2) { A[0] = 0.5; t[0] = 0.5; }
    else if (stages == 2 && order == 2) {
        const double g = 1.0 - 1.0 / std::sqrt(2.0);
        A[0] = g; A[1] = 1.0 - g; A[3] = g;            // A[i + 2j]
        t[0] = g; t[1] = 1.0;
    } else if (stages == 2 && order == 3) {
        const double g = (3.0 + std::sqrt(3.0)) / 6.0;
        A[0] = g; A[1] = 1.0 - 2.0 * g; A[3] = g;
        t[0] = g; t[1] = 1.0 - g;
    } else if (stages == 3 && order == 3) {
        double g = 0.4358665;                             // Newton on g^3 - 3g^2 + 3g/2 - 1/6
        for (int it = 0; it < 50; it++) g -= (g * g * g - 3 * g * g + 1.5 * g - 1.0 / 6.0) / (3 * g * g - 6 * g + 1.5);
        const double t2 = 0.5 * (1.0 + g);
        const double b1 = -(6 * g * g - 16 * g + 1) / 4.0, b2 = (6 * g * g - 20 * g + 5) / 4.0;
        A[0] = g; A[1] = t2 - g; A[2] = b1;               // A[i + 3j]
        A[4] = g; A[5] = b2; A[8] = g;
        t[0] = g; t[1] = t2; t[2] = 1.0;
    } else {
        return false;
    }
    // inverse of the lower-triangular A, column by column
    const int s = stages;
    for (int j = 0; j < s; j++)
        for (int i = 0; i < s; i++) {
            double v = 0.0;
            if (i == j) v = 1.0 / A[i + s * i];
            else if (i > j) {
                double acc = 0.0;
                for (int k = j; k < i; k++) acc += A[i + s * k] * d[k + s * j];
                v = -acc / A[i + s * i];
            }
            d[i + s * j] = v;
        }
    return true;
}

// sh = cu_i udgi + cu udg + cs sh on the u components, 0 on the q components.
__global__ void dirk_source_kernel(long long n, int npv, int nc, int ncu, double ci, double cu, double cs,
                                   const double* __restrict__ udgi, const double* __restrict__ udg,
                                   double* __restrict__ sh) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int comp = (int)((i / npv) % nc);
        sh[i] = (comp < ncu) ? ci * udgi[i] + cu * udg[i] + cs * sh[i] : 0.0;
    }
}

}  // namespace

extern "C" {

int hfem_create(const hfem_dims* dims, int device, hfem_ctx** out) {
    if (!dims || !out) return HFEM_E_ARG;
    *out = nullptr;
    hfem_ctx* c = new hfem_ctx();
    c->dims = *dims;
    c->device = device;
    const hfem_dims& d = *dims;
    if (d.nd < 2 || d.nd > 3 || d.nfe != d.nd + 1 || d.ne <= 0 || d.nf <= 0 || d.nblocks < d.nf) {
        delete c;
        return HFEM_E_ARG;
    }
    for (const Launch& L : launches())
        if (L.nd == d.nd && L.npv == d.npv && L.npf == d.npf && L.ngv == d.ngv && L.ngf == d.ngf) c->L = &L;
    if (!c->L) {
        delete c;
        return HFEM_E_UNSUPPORTED;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        delete c;
        return HFEM_E_CUDA;
    }
    c->ncu = d.nd + 2;
    c->nc = c->ncu * (d.nd + 1);
    c->nch = c->ncu;
    c->ndf = d.npf * d.nfe;
    c->n = d.npv * c->ncu;
    c->nb = c->nch * c->ndf;
    c->bsz = c->nch * d.npf;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return HFEM_E_CUDA;
    }
    c->stream = c->own;
    const Launch& L = *c->L;
    cudaFuncSetAttribute(L.elem_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.elem_smem);
    for (int t = 0; t < 2; t++)
        for (int g = 0; g < 2; g++)
            cudaFuncSetAttribute(L.elem_fn_v[t][g], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.elem_smem);
    cudaFuncSetAttribute(L.q_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.q_smem);
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L.elem_fn, NT, L.elem_smem);
    c->grid_elem = std::max(1, std::min(d.ne, sms(device) * std::max(occ, 1)));
    // the workspace has grid_elem slots: no variant runs more CTAs
    for (int t = 0; t < 2; t++)
        for (int g = 0; g < 2; g++) {
            occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L.elem_fn_v[t][g], NT, L.elem_smem);
            c->grid_elem_v[t][g] = std::max(1, std::min(c->grid_elem, sms(device) * std::max(occ, 1)));
        }
    cudaFuncSetAttribute(L.g1.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.g1.smem);
    cudaFuncSetAttribute(L.g2.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.g2.smem);
    cudaFuncSetAttribute(L.tc_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.tc_smem);
    cudaFuncSetAttribute(L.fused_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.fused_smem);
    for (const GemmLaunch& g : gemm_candidates())
        cudaFuncSetAttribute(g.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem);
    occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L.tc_fn, TC_THREADS, L.tc_smem);
    // the CTAs resident on an SM share its 512 tensor-memory columns
    c->grid_tc = std::max(1, std::min(d.ne, sms(device) * std::max(1, std::min(occ, 512 / L.tc_tmem))));
    occ = 0;
    cudaFuncSetAttribute(L.inv_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.inv_smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L.inv_fn, L.inv_threads, L.inv_smem);
    c->grid_inv = std::max(1, std::min(d.ne, sms(device) * std::max(occ, 1)));
    if (pool_alloc(device, (void**)&c->rnorm, sizeof(double)) != cudaSuccess) {
        cudaStreamDestroy(c->own);
        delete c;
        return HFEM_E_NOMEM;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->own);
        delete c;
        return HFEM_E_CUDA;
    }
    *out = c;
    return 0;
}

int hfem_destroy(hfem_ctx* c) {
    if (!c) return HFEM_E_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    void* ptrs[] = {c->shapvt, c->shapvg, c->svsv, c->shapft, c->shapfg, c->sfsf, c->perm, c->dgnodes, c->elcon,
                    c->rowstart, c->colidx, c->blk_src, c->face_src, c->rowface, c->colface, c->udg, c->uh, c->sh,
                    c->D, c->F, c->K, c->H, c->Ru, c->DinvRu, c->Rh, c->Ro, c->ru2, c->Hg, c->Rg, c->Rr, c->rnorm, c->ws, c->DinvF,
                    c->info, c->Minv, c->V, c->w, c->x, c->pb, c->scal, c->part, c->binfo, c->udgi,
                    c->eprob, c->fprob, c->pparam, c->palpha, c->seg_pstart, c->seg_pseg, c->seg_p0,
                    c->seg_ticket, c->seg_part, c->seg_partk, c->seg_h, c->seg_y, c->seg_nrm, c->seg_act, c->seg_k, c->tc_err, c->rn_part, c->bf, c->bcm, c->bcs, c->Minv32,
                    c->d_u2o, c->d_rows_lo, c->d_rows_up, c->d_fptr, c->d_fpos, c->Mg, c->bl_t, c->bl_y,
                    c->d_lvl_lo, c->d_lvl_up, c->Mg32, c->d_frec, c->d_lrec, c->d_urec, c->gm_H, c->gm_cs, c->gm_sn, c->gm_g, c->gm_nrmb, c->gm_hist,
                    c->gm_state, c->gm_its, c->gm_jc};
    for (void* p : ptrs)
        if (p) pool_free(p);
    for (auto& p : c->timer.pending) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    if (c->bilu_exec) cudaGraphExecDestroy(c->bilu_exec);
    for (cudaEvent_t ev : c->chunk_ev) cudaEventDestroy(ev);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return 0;
}

const char* hfem_last_error(const hfem_ctx* c) { return c ? c->err.c_str() : "null context"; }

int hfem_set_stream(hfem_ctx* c, void* stream) {
    if (!c) return HFEM_E_ARG;
    c->stream = stream ? (cudaStream_t)stream : c->own;
    return 0;
}

int hfem_set_master(hfem_ctx* c, const double* shapvt, const double* shapvg, const double* svsv, const double* shapft,
                    const double* shapfg, const double* sfsf, const int* perm) {
    if (!c || !shapvt || !shapvg || !svsv || !shapft || !shapfg || !sfsf || !perm) return HFEM_E_ARG;
    const hfem_dims& d = c->dims;
    for (int i = 0; i < d.npf * d.nfe; i++)
        if (perm[i] < 0 || perm[i] >= d.npv) return fail(c, HFEM_E_ARG, "perm[%d] = %d out of range", i, perm[i]);
    int rc;
    CK(cudaSetDevice(c->device));
    const size_t v1 = (size_t)d.ngv * d.npv * (d.nd + 1), v2 = (size_t)d.npv * d.npv * d.ngv * (d.nd + 1);
    const size_t f1 = (size_t)d.ngf * d.npf * d.nd, f2 = (size_t)d.npf * d.npf * d.ngf * d.nd;
    if ((rc = upload(c, &c->shapvt, shapvt, v1)) || (rc = upload(c, &c->shapvg, shapvg, v1)) ||
        (rc = upload(c, &c->svsv, svsv, v2)) || (rc = upload(c, &c->shapft, shapft, f1)) ||
        (rc = upload(c, &c->shapfg, shapfg, f1)) || (rc = upload(c, &c->sfsf, sfsf, f2)) ||
        (rc = upload(c, &c->perm, perm, (size_t)d.npf * d.nfe)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->have_master = true;
    return 0;
}

int hfem_set_mesh(hfem_ctx* c, const double* dgnodes, const int* elcon, const int* t2f, const int* rowstart,
                  const int* colidx) {
    if (!c || !dgnodes || !elcon || !t2f || !rowstart || !colidx) return HFEM_E_ARG;
    const hfem_dims& d = c->dims;
    const int ne = d.ne, nf = d.nf, nfe = d.nfe, npf = d.npf, ndf = c->ndf, nblk = d.nblocks;
    // connectivity checks (the reference's own invariants: digasopre.m:80-88, globalassembly.cpp:69-75)
    if (rowstart[0] != 0 || rowstart[nf] != nblk) return fail(c, HFEM_E_MESH, "ent2entStart must run from 0 to nblocks");
    for (int i = 0; i < nf; i++) {
        if (rowstart[i + 1] <= rowstart[i]) return fail(c, HFEM_E_MESH, "empty CSR row %d", i);
        if (colidx[rowstart[i]] != i) return fail(c, HFEM_E_MESH, "row %d does not start with its diagonal block", i);
    }
    for (int k = 0; k < nblk; k++)
        if (colidx[k] < 0 || colidx[k] >= nf) return fail(c, HFEM_E_MESH, "ent2ent[%d] out of range", k);
    std::vector<int> rowface(nblk), blk((size_t)nblk * 6, -1), fsrc((size_t)nf * 4, -1), fcount(nf, 0), bcount(nblk, 0);
    for (int i = 0; i < nf; i++)
        for (int k = rowstart[i]; k < rowstart[i + 1]; k++) rowface[k] = i;
    for (int e = 0; e < ne; e++) {
        for (int a = 0; a < nfe; a++) {
            const int i = t2f[e * nfe + a];
            if (i < 0 || i >= nf) return fail(c, HFEM_E_MESH, "t2f of element %d out of range", e);
            for (int m = 0; m < npf; m++) {
                const int g = elcon[(size_t)e * ndf + a * npf + m];
                if (g < i * npf || g >= (i + 1) * npf)
                    return fail(c, HFEM_E_MESH, "elcon of element %d face %d does not lie on face %d", e, a, i);
            }
            if (fcount[i] >= 2) return fail(c, HFEM_E_MESH, "face %d has more than two elements", i);
            fsrc[(i * 2 + fcount[i]) * 2 + 0] = e;
            fsrc[(i * 2 + fcount[i]) * 2 + 1] = a;
            fcount[i]++;
            for (int b = 0; b < nfe; b++) {
                const int j = t2f[e * nfe + b];
                int k = -1;
                for (int kk = rowstart[i]; kk < rowstart[i + 1]; kk++)
                    if (colidx[kk] == j) { k = kk; break; }
                if (k < 0) return fail(c, HFEM_E_MESH, "block (%d, %d) of element %d missing from the CSR", i, j, e);
                if (bcount[k] >= 2)
                    return fail(c, HFEM_E_MESH, "block (%d, %d) receives more than two element contributions", i, j);
                blk[(k * 2 + bcount[k]) * 3 + 0] = e;
                blk[(k * 2 + bcount[k]) * 3 + 1] = a;
                blk[(k * 2 + bcount[k]) * 3 + 2] = b;
                bcount[k]++;
            }
        }
    }
    int rc;
    CK(cudaSetDevice(c->device));
    std::vector<int> colface(colidx, colidx + nblk);
    if ((rc = upload(c, &c->dgnodes, dgnodes, (size_t)ne * d.npv * d.nd)) ||
        (rc = upload(c, &c->elcon, elcon, (size_t)ne * ndf)) || (rc = upload(c, &c->rowstart, rowstart, (size_t)nf + 1)) ||
        (rc = upload(c, &c->colidx, colidx, (size_t)nblk)) || (rc = upload(c, &c->blk_src, blk.data(), blk.size())) ||
        (rc = upload(c, &c->face_src, fsrc.data(), fsrc.size())) ||
        (rc = upload(c, &c->rowface, rowface.data(), rowface.size())) ||
        (rc = upload(c, &c->colface, colface.data(), colface.size())))
        return rc;
    if ((rc = dalloc(c, &c->Hg, (size_t)nblk * c->bsz * c->bsz)) || (rc = dalloc(c, &c->Rg, (size_t)nf * c->bsz)) ||
        (rc = dalloc(c, &c->Rr, (size_t)nf * c->bsz)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->h_rowstart.assign(rowstart, rowstart + nf + 1);
    c->h_colidx.assign(colidx, colidx + nblk);
    c->have_order = false;
    if (c->bf) { pool_free(c->bf); c->bf = nullptr; }      // boundary flags belong to the old mesh
    c->have_mesh = true;
    return 0;
}

int hfem_set_boundary(hfem_ctx* c, const int* bf, int nbnd, const int* bcm, const double* bcs) {
    if (!c || !bf || nbnd < 0 || (nbnd > 0 && (!bcm || !bcs))) return HFEM_E_ARG;
    if (!c->have_mesh) return fail(c, HFEM_E_STATE, "set the mesh before its boundary");
    const hfem_dims& d = c->dims;
    for (int b = 0; b < nbnd; b++)
        if (bcm[b] != 1 && bcm[b] != 2 && bcm[b] != 5 && bcm[b] != 6 && bcm[b] != 7)
            return fail(c, HFEM_E_UNSUPPORTED, "boundary condition type %d (supported: 1, 2, 5, 6, 7)", bcm[b]);
    // a boundary face belongs to one element, an interior one to two
    std::vector<int> fsrc((size_t)d.nf * 4);
    CK(cudaMemcpy(fsrc.data(), c->face_src, sizeof(int) * fsrc.size(), cudaMemcpyDeviceToHost));
    int any = 0;
    for (int e = 0; e < d.ne; e++)
        for (int a = 0; a < d.nfe; a++) {
            const int v = bf[(size_t)e * d.nfe + a];
            if (v < 0) {
                if (-v - 1 >= nbnd) return fail(c, HFEM_E_ARG, "bf of element %d face %d names boundary %d", e, a, -v - 1);
                any = 1;
            }
        }
    for (int f = 0; f < d.nf; f++) {
        const bool two = fsrc[(f * 2 + 1) * 2] >= 0;
        const int e = fsrc[(f * 2) * 2], a = fsrc[(f * 2) * 2 + 1];
        const bool bnd = bf[(size_t)e * d.nfe + a] < 0;
        if (bnd == two) return fail(c, HFEM_E_MESH, "face %d: boundary flag and element count disagree", f);
    }
    int rc;
    CK(cudaSetDevice(c->device));
    if (!any) {
        if (c->bf) { pool_free(c->bf); c->bf = nullptr; }
        c->nbnd = 0;
        return 0;
    }
    if ((rc = upload(c, &c->bf, bf, (size_t)d.ne * d.nfe)) || (rc = upload(c, &c->bcm, bcm, (size_t)nbnd)) ||
        (rc = upload(c, &c->bcs, bcs, (size_t)nbnd * c->nch)))
        return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->nbnd = nbnd;
    c->assembled = false;
    return 0;
}

int hfem_set_app(hfem_ctx* c, int appname) {
    if (!c) return HFEM_E_ARG;
    if (appname != 0 && appname != 1)
        return fail(c, HFEM_E_UNSUPPORTED, "appname %d (supported: 0 Euler, 1 Navier-Stokes)", appname);
    c->appname = appname;
    c->assembled = false;
    return 0;
}

int hfem_set_models(hfem_ctx* c, int conv_stab, int viscosity_model) {
    if (!c) return HFEM_E_ARG;
    if (conv_stab < 0 || conv_stab > 2)
        return fail(c, HFEM_E_UNSUPPORTED, "convStabMethod %d (supported: 0 constant, 1 Lax-Friedrichs, 2 Roe)",
                    conv_stab);
    if (viscosity_model < 0 || viscosity_model > 1)
        return fail(c, HFEM_E_UNSUPPORTED, "viscosityModel %d (supported: 0 constant, 1 Sutherland)", viscosity_model);
    c->conv_stab = conv_stab;
    c->visc_model = viscosity_model;
    c->assembled = false;
    return 0;
}

int hfem_set_physics(hfem_ctx* c, const double* param, int tdep, double fc_u, double fc_q, double time) {
    if (!c || !param) return HFEM_E_ARG;
    if (!(param[0] > 1.0) || !(param[2] > 0.0) || !(param[3] > 0.0))
        return fail(c, HFEM_E_ARG, "physicsparam needs gamma > 1, Re > 0, Pr > 0");
    for (int i = 0; i < 6; i++) c->param[i] = param[i];
    c->tdep = tdep;
    c->fc_u = fc_u;
    c->fc_q = fc_q;
    c->time = time;
    c->have_phys = true;
    return 0;
}

static int set_solution_common(hfem_ctx* c, const double* udg, const double* uh, const double* sh, cudaMemcpyKind kind) {
    if (!c || !udg || !uh) return HFEM_E_ARG;
    const hfem_dims& d = c->dims;
    const size_t nudg = (size_t)d.ne * d.npv * c->nc, nuh = (size_t)d.nf * c->bsz;
    int rc;
    CK(cudaSetDevice(c->device));
    if (!c->udg) {
        if ((rc = dalloc(c, &c->udg, nudg)) || (rc = dalloc(c, &c->uh, nuh)) || (rc = dalloc(c, &c->sh, nudg))) return rc;
    }
    CK(cudaMemcpyAsync(c->udg, udg, sizeof(double) * nudg, kind, c->stream));
    CK(cudaMemcpyAsync(c->uh, uh, sizeof(double) * nuh, kind, c->stream));
    if (sh) CK(cudaMemcpyAsync(c->sh, sh, sizeof(double) * nudg, kind, c->stream));
    else CK(cudaMemsetAsync(c->sh, 0, sizeof(double) * nudg, c->stream));
    c->have_sol = true;
    c->assembled = false;
    return 0;
}

int hfem_set_solution(hfem_ctx* c, const double* udg, const double* uh, const double* sh) {
    int rc = set_solution_common(c, udg, uh, sh, cudaMemcpyHostToDevice);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int hfem_assemble_host(hfem_ctx* c, const double* udg, const double* uh, const double* sh, int chunks,
                       double* rnorm) {
    if (!c || !udg || !uh || chunks < 1) return c ? fail(c, HFEM_E_ARG, "null array or chunks < 1") : HFEM_E_ARG;
    const hfem_dims& d = c->dims;
    const size_t per_e = (size_t)d.npv * c->nc, nuh = (size_t)d.nf * c->bsz;
    chunks = std::max(1, std::min(chunks, d.ne));
    int rc;
    CK(cudaSetDevice(c->device));
    if (!c->udg) {
        if ((rc = dalloc(c, &c->udg, d.ne * per_e)) || (rc = dalloc(c, &c->uh, nuh)) ||
            (rc = dalloc(c, &c->sh, d.ne * per_e)))
            return rc;
    }
    if (!c->copy_stream) CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    while ((int)c->chunk_ev.size() < chunks + 1) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        c->chunk_ev.push_back(ev);
    }
    // the copies overwrite the state only after the work queued before them
    CK(cudaEventRecord(c->chunk_ev[0], c->stream));
    CK(cudaStreamWaitEvent(c->copy_stream, c->chunk_ev[0], 0));
    CK(cudaMemcpyAsync(c->uh, uh, sizeof(double) * nuh, cudaMemcpyHostToDevice, c->copy_stream));
    c->chunk_lo.assign(chunks + 1, 0);
    for (int k = 0; k < chunks; k++) {
        const int e0 = (int)((long long)d.ne * k / chunks), e1 = (int)((long long)d.ne * (k + 1) / chunks);
        c->chunk_lo[k] = e0;
        c->chunk_lo[k + 1] = e1;
        const size_t off = (size_t)e0 * per_e, cnt = (size_t)(e1 - e0) * per_e;
        CK(cudaMemcpyAsync(c->udg + off, udg + off, sizeof(double) * cnt, cudaMemcpyHostToDevice, c->copy_stream));
        if (sh) CK(cudaMemcpyAsync(c->sh + off, sh + off, sizeof(double) * cnt, cudaMemcpyHostToDevice, c->copy_stream));
        else CK(cudaMemsetAsync(c->sh + off, 0, sizeof(double) * cnt, c->copy_stream));
        CK(cudaEventRecord(c->chunk_ev[k + 1], c->copy_stream));
    }
    c->pending_chunks = chunks;
    c->have_sol = true;
    c->assembled = false;
    rc = run_assembly(c, true, rnorm);
    if (rc) {
        c->pending_chunks = 0;
        cudaStreamSynchronize(c->copy_stream);
    }
    return rc;
}

int hfem_set_solution_device(hfem_ctx* c, const double* udg, const double* uh, const double* sh) {
    return set_solution_common(c, udg, uh, sh, cudaMemcpyDeviceToDevice);
}

int hfem_get_solution(hfem_ctx* c, double* udg, double* uh) {
    if (!c || !c->have_sol) return c ? fail(c, HFEM_E_STATE, "no solution set") : HFEM_E_ARG;
    const size_t nudg = (size_t)c->dims.ne * c->dims.npv * c->nc, nuh = (size_t)c->dims.nf * c->bsz;
    if (udg) CK(cudaMemcpyAsync(udg, c->udg, sizeof(double) * nudg, cudaMemcpyDeviceToHost, c->stream));
    if (uh) CK(cudaMemcpyAsync(uh, c->uh, sizeof(double) * nuh, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int hfem_getq(hfem_ctx* c) {
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = launch_getq(c, nullptr, 0.0))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    flush_timer(c);
    c->assembled = false;
    return 0;
}

int hfem_assemble(hfem_ctx* c, double* rnorm) { return run_assembly(c, true, rnorm); }

int hfem_residual(hfem_ctx* c, double* rnorm) { return run_assembly(c, false, rnorm); }

int hfem_gmres(hfem_ctx* c, int precond, int restart, double tol, int maxit, int* conv, int* iters, double* hist,
               int hist_len) {
    if (!c) return HFEM_E_ARG;
    return gmres_impl(c, precond, restart, tol, maxit, conv, iters, hist, hist_len);
}

int hfem_update(hfem_ctx* c, double alpha) {
    if (!c) return HFEM_E_ARG;
    return update_impl(c, alpha);
}

// solveNonlinearProblem (solvers/dgsolvers.cpp:106-205), damped Newton with the
// reference's line search: halve alpha (stepping back from the previous trial)
// while the residual grows, down to alphaMin = 1e-4.
int hfem_newton(hfem_ctx* c, double newton_tol, int newton_maxiter, int precond, int restart, double gmres_tol,
                int gmres_maxit, double* hist, int hist_len, int* niter, int* converged) {
    if (!c) return HFEM_E_ARG;
    int rc = ready(c);
    if (rc) return rc;
    const double alphaMin = 1.0e-4;
    double rNorm = newton_tol + 1.0;
    int iter = 0, nh = 0, robust = 0;
    while (rNorm > newton_tol && iter < newton_maxiter) {
        iter++;
        double oldNorm = 0.0;
        if ((rc = run_assembly(c, true, &oldNorm))) return rc;
        if (hist && nh < hist_len) hist[nh++] = oldNorm;
        if (std::isnan(oldNorm) || std::isinf(oldNorm))
            return fail(c, HFEM_E_SINGULAR, "residual norm of Newton iterate %d is NaN or Inf", iter);
        int conv = 0, its = 0;
        if ((rc = gmres_impl(c, precond, restart, gmres_tol, gmres_maxit, &conv, &its, nullptr, 0))) return rc;
        if (conv == -1) break;
        if (iter == 1 && oldNorm < newton_tol) {
            rNorm = oldNorm;
            break;
        }
        double alpha = 1.0;
        while (true) {
            if ((rc = update_impl(c, alpha))) return rc;
            if ((rc = run_assembly(c, false, &rNorm))) return rc;
            if (std::isnan(rNorm) || std::isinf(rNorm) || (rNorm > oldNorm && rNorm > newton_tol)) {
                const double a = std::fabs(alpha / 2);
                alpha = -a;
                if (a < alphaMin) {
                    if (robust == 0) {
                        robust = 1;
                        alpha = -2.0 * std::fabs(alpha);
                        if ((rc = update_impl(c, alpha))) return rc;
                    }
                    break;
                }
            } else {
                break;
            }
        }
    }
    if (hist && nh < hist_len) hist[nh++] = rNorm;
    if (niter) *niter = iter;
    if (converged) *converged = rNorm < newton_tol ? 1 : 0;
    return 0;
}

// One time step of solveUnsteadyProblem (solvers/dgsolvers.cpp:221-444): for
// each DIRK stage set time = t + dt c_i, fc_u = d_ii/dt, fc_q = 1, form the
// stage source SH from the step's initial state and the previous stage
// (dgsolvers.cpp:319-348, q part zeroed) and solve the stage with the Newton
// driver.  A stage that does not converge returns HFEM_E_SINGULAR (the
// reference calls error() and exits).
int hfem_dirk_step(hfem_ctx* c, double dt, int stages, int order, double newton_tol, int newton_maxiter,
                   int precond, int restart, double gmres_tol, int gmres_maxit, int* newton_iters) {
    if (!c) return HFEM_E_ARG;
    int rc = ready(c);
    if (rc) return rc;
    double d[9], t[3];
    if (!(dt > 0.0) || !dirk_table(stages, order, d, t))
        return fail(c, HFEM_E_ARG, "unsupported DIRK(%d,%d) or dt <= 0", stages, order);
    const hfem_dims& dm = c->dims;
    const long long n = (long long)dm.ne * dm.npv * c->nc;
    if (!c->udgi && (rc = dalloc(c, &c->udgi, (size_t)n))) return rc;
    CK(cudaMemcpyAsync(c->udgi, c->udg, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    const int S = stages;
    const double t0 = c->time;
    int total_iters = 0;
    for (int s = 0; s < S; s++) {
        double ci = 0.0, cu = 0.0, cs = 0.0;
        if (s == 0) {
            ci = d[0] / dt;
        } else if (s == 1) {
            ci = (d[1] + d[S + 1]) / dt;
            cu = -d[1] / dt;
        } else {
            const double r = d[2] / d[1];
            ci = (d[2] + d[S + 2] + d[2 * S + 2]) / dt - r * (d[1] + d[S + 1]) / dt;
            cs = r;
            cu = -d[S + 2] / dt;
        }
        dirk_source_kernel<<<sms(c->device) * 4, 256, 0, c->stream>>>(n, dm.npv, c->nc, c->ncu, ci, cu, cs, c->udgi,
                                                                      c->udg, c->sh);
        if ((rc = check_launch(c, "dirk_source"))) return rc;
        c->time = t0 + dt * t[s];
        c->fc_u = d[s + S * s] / dt;
        c->fc_q = 1.0;
        c->tdep = 1;
        int it = 0, conv = 0;
        if ((rc = hfem_newton(c, newton_tol, newton_maxiter, precond, restart, gmres_tol, gmres_maxit, nullptr, 0,
                              &it, &conv)))
            return rc;
        total_iters += it;
        if (!conv) {
            c->time = t0;
            return fail(c, HFEM_E_SINGULAR, "DIRK stage %d did not converge in %d Newton iterations", s + 1, it);
        }
    }
    c->time = t0 + dt;
    if (newton_iters) *newton_iters = total_iters;
    return 0;
}

// Several independent problems packed into this context's mesh (a disjoint
// union: no face is shared between problems).  eprob: element -> problem,
// fprob: face -> problem, params: per problem [gamma, eps, Re, Pr, Mach, tau,
// tdep, fc_u].  The element kernels then read each element's own physics.
int hfem_set_problem_map(hfem_ctx* c, int nprob, const int* eprob, const int* fprob, const double* params) {
    if (!c || nprob < 1 || !eprob || !fprob || !params) return HFEM_E_ARG;
    const hfem_dims& d = c->dims;
    for (int e = 0; e < d.ne; e++)
        if (eprob[e] < 0 || eprob[e] >= nprob) return fail(c, HFEM_E_ARG, "eprob[%d] out of range", e);
    for (int f = 0; f < d.nf; f++)
        if (fprob[f] < 0 || fprob[f] >= nprob) return fail(c, HFEM_E_ARG, "fprob[%d] out of range", f);
    int rc;
    CK(cudaSetDevice(c->device));
    if ((rc = upload(c, &c->eprob, eprob, (size_t)d.ne)) || (rc = upload(c, &c->fprob, fprob, (size_t)d.nf)) ||
        (rc = upload(c, &c->pparam, params, (size_t)nprob * 8)) || (rc = dalloc(c, &c->palpha, (size_t)nprob)))
        return rc;
    // Krylov segments (hfem_gmres_problems): when fprob is non-decreasing and
    // every problem owns a face, problem p's slice of the trace vector is one
    // contiguous segment, cut into pieces of <= SEG_PIECE entries.
    c->npieces = 0;
    c->seg_single = false;
    bool sorted = true;
    std::vector<int> fcount(nprob, 0);
    for (int f = 0; f < d.nf; f++) {
        fcount[fprob[f]]++;
        if (f && fprob[f] < fprob[f - 1]) sorted = false;
    }
    for (int p = 0; p < nprob; p++) sorted = sorted && fcount[p] > 0;
    if (sorted) {
        // piece length: a power of two in [1024, SEG_PIECE] giving about 4 CTAs per SM
        const long long ntot = (long long)d.nf * c->bsz;
        long long piece = 1024;
        while (piece < SEG_PIECE && piece * 4 * sms(c->device) < ntot) piece *= 2;
        std::vector<long long> pstart;
        std::vector<int> pseg, p0(nprob + 1);
        long long a = 0;
        for (int p = 0; p < nprob; p++) {
            p0[p] = (int)pseg.size();
            const long long b = a + (long long)fcount[p] * c->bsz;
            for (long long s = a; s < b; s += piece) {
                pstart.push_back(s);
                pseg.push_back(p);
            }
            a = b;
        }
        p0[nprob] = (int)pseg.size();
        pstart.push_back(a);
        c->npieces = (int)pseg.size();
        if ((rc = upload(c, &c->seg_pstart, pstart.data(), pstart.size())) ||
            (rc = upload(c, &c->seg_pseg, pseg.data(), pseg.size())) ||
            (rc = upload(c, &c->seg_p0, p0.data(), p0.size())) || (rc = dalloc(c, &c->seg_ticket, (size_t)nprob)) ||
            (rc = dalloc(c, &c->seg_part, pseg.size())) || (rc = dalloc(c, &c->seg_nrm, (size_t)2 * nprob)) ||
            (rc = dalloc(c, &c->seg_act, (size_t)nprob)) || (rc = dalloc(c, &c->seg_k, (size_t)nprob)))
            return rc;
        CK(cudaMemsetAsync(c->seg_ticket, 0, sizeof(int) * nprob, c->stream));
        c->seg_restart = 0;
    }
    CK(cudaStreamSynchronize(c->stream));
    c->nprob = nprob;
    return 0;
}

// Per-problem residual norms of the last assembly or residual pass:
// rnorm[p] = sqrt(sum over p's elements ||Ru_e||^2 + ||Rr restricted to p's faces||^2).
int hfem_problem_rnorms(hfem_ctx* c, double* rnorm) {
    if (!c || !rnorm) return HFEM_E_ARG;
    if (!c->nprob || !c->ru2) return fail(c, HFEM_E_STATE, "no problem map or no residual yet");
    const hfem_dims& d = c->dims;
    std::vector<double> ru2(d.ne), rr((size_t)d.nf * c->bsz);
    std::vector<int> ep(d.ne), fp(d.nf);
    CK(cudaMemcpyAsync(ru2.data(), c->ru2, sizeof(double) * ru2.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(rr.data(), c->Rr, sizeof(double) * rr.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(ep.data(), c->eprob, sizeof(int) * ep.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(fp.data(), c->fprob, sizeof(int) * fp.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<double> acc(c->nprob, 0.0);
    for (int e = 0; e < d.ne; e++) acc[ep[e]] += ru2[e];
    for (int f = 0; f < d.nf; f++)
        for (int k = 0; k < c->bsz; k++) acc[fp[f]] += rr[(size_t)f * c->bsz + k] * rr[(size_t)f * c->bsz + k];
    for (int p = 0; p < c->nprob; p++) rnorm[p] = std::sqrt(acc[p]);
    return 0;
}

// updateSol with a step length per problem: uh += alpha_p x, u += alpha_p (D^-1 Ru - D^-1 F x_e).
int hfem_update_problems(hfem_ctx* c, const double* alpha) {
    if (!c || !alpha) return HFEM_E_ARG;
    if (!c->nprob) return fail(c, HFEM_E_STATE, "no problem map");
    if (!c->assembled || !c->x) return fail(c, HFEM_E_STATE, "assemble and solve before update");
    int rc;
    CK(cudaMemcpyAsync(c->palpha, alpha, sizeof(double) * c->nprob, cudaMemcpyHostToDevice, c->stream));
    axpy_prob_kernel<<<sms(c->device) * 4, 256, 0, c->stream>>>(nvec(c), c->bsz, c->fprob, c->palpha, c->x, c->uh);
    if ((rc = check_launch(c, "uh update"))) return rc;
    c->palpha_on = true;
    rc = launch_getq(c, c->x, 0.0);
    c->palpha_on = false;
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    flush_timer(c);
    return 0;
}

int hfem_assemble_async(hfem_ctx* c) {
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = ensure_assembly_buffers(c))) return rc;
    return enqueue_assembly(c, true);
}

int hfem_assemble_finish(hfem_ctx* c, double* rnorm) {
    if (!c) return HFEM_E_ARG;
    return finish_assembly(c, true, rnorm);
}

int hfem_gemm_candidates(void) { return (int)gemm_candidates().size(); }

int hfem_set_gemm_tiles(hfem_ctx* c, int g1, int g2) {
    if (!c) return HFEM_E_ARG;
    const int nc = (int)gemm_candidates().size();
    if (g1 < -1 || g1 >= nc || g2 < -1 || g2 >= nc) return fail(c, HFEM_E_ARG, "tiling index out of range");
    c->g1_sel = g1;
    c->g2_sel = g2;
    return 0;
}

// Time every batched-GEMM tiling on this context's own operands (reps
// launches each, CUDA events on the context's stream) and keep the fastest
// for D^-1 F and for the Schur update.  The condensed blocks are overwritten
// while timing, so the context must be assembled again before it is used.
int hfem_autotune(hfem_ctx* c, int reps, int* best, double* ms) {
    if (!c || reps < 1) return HFEM_E_ARG;
    int rc = ready(c);
    if (rc) return rc;
    if ((rc = ensure_assembly_buffers(c))) return rc;
    const bool timing = c->timer.on;
    c->timer.on = false;
    if ((rc = enqueue_assembly(c, true))) return rc;
    if ((rc = finish_assembly(c, true, nullptr))) return rc;
    const int ne = c->dims.ne, n = c->n, nb = c->nb;
    const auto& cand = gemm_candidates();
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double bt[2] = {1e300, 1e300};
    int bi[2] = {-1, -1};
    for (int which = 0; which < 2; which++)
        for (size_t k = 0; k < cand.size(); k++) {
            const GemmLaunch& g = cand[k];
            auto launch = [&]() {
                if (which == 0)
                    g.run(c->stream, ne, n, nb, n, 1.0, c->D, n, (long long)n * n, c->F, n, (long long)n * nb, 0.0,
                          c->DinvF, n, (long long)n * nb);
                else
                    g.run(c->stream, ne, nb, nb, n, -1.0, c->K, nb, (long long)nb * n, c->DinvF, n,
                          (long long)n * nb, 1.0, c->H, nb, (long long)nb * nb);
            };
            launch();                                      // warm-up
            if ((rc = check_launch(c, "autotune"))) return rc;
            CK(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < reps; r++) launch();
            CK(cudaEventRecord(e1, c->stream));
            CK(cudaEventSynchronize(e1));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, e0, e1));
            const double per = (double)t / reps;
            if (ms) ms[which * cand.size() + k] = per;
            if (per < bt[which]) bt[which] = per, bi[which] = (int)k;
        }
    // the fused kernel does both products: kept when it beats the best pair
    {
        c->L->schur_fused(c->stream, ne, c->D, c->F, c->K, c->H, c->DinvF);   // warm-up
        if ((rc = check_launch(c, "autotune"))) return rc;
        CK(cudaEventRecord(e0, c->stream));
        for (int r = 0; r < reps; r++) c->L->schur_fused(c->stream, ne, c->D, c->F, c->K, c->H, c->DinvF);
        CK(cudaEventRecord(e1, c->stream));
        CK(cudaEventSynchronize(e1));
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, e0, e1));
        if ((double)t / reps <= bt[0] + bt[1]) bi[0] = bi[1] = -1;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->g1_sel = bi[0];
    c->g2_sel = bi[1];
    c->assembled = false;
    c->timer.on = timing;
    if (best) best[0] = bi[0], best[1] = bi[1];
    return 0;
}

struct hfem_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;
};

// One CUDA graph holding the assembly of several contexts (e.g. one per
// element shape), each on its own branch so they run concurrently.
int hfem_graph_capture(hfem_ctx** ctxs, int n, void* stream, hfem_graph** out) {
    if (!ctxs || n < 1 || !stream || !out) return HFEM_E_ARG;
    hfem_ctx* c0 = ctxs[0];
    hfem_ctx* c = c0;
    for (int i = 0; i < n; i++) {
        if (!ctxs[i] || ctxs[i]->device != c0->device) return fail(c0, HFEM_E_ARG, "contexts must share a device");
        int rc = ready(ctxs[i]);
        if (rc) return rc;
        if ((rc = ensure_assembly_buffers(ctxs[i]))) return rc;
        CK(cudaStreamSynchronize(ctxs[i]->stream));
    }
    CK(cudaSetDevice(c0->device));
    auto* g = new hfem_graph();
    g->side.resize(n);
    g->ev.resize(n + 1);
    for (int i = 0; i < n; i++) CK(cudaStreamCreateWithFlags(&g->side[i], cudaStreamNonBlocking));
    for (int i = 0; i <= n; i++) CK(cudaEventCreateWithFlags(&g->ev[i], cudaEventDisableTiming));
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<cudaStream_t> saved(n);
    std::vector<bool> timing(n);
    int rc = 0;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(g->ev[n], s);
    for (int i = 0; i < n && !rc; i++) {
        saved[i] = ctxs[i]->stream;
        timing[i] = ctxs[i]->timer.on;
        ctxs[i]->timer.on = false;
        ctxs[i]->stream = g->side[i];
        cudaStreamWaitEvent(g->side[i], g->ev[n], 0);
        rc = enqueue_assembly(ctxs[i], true);
        cudaEventRecord(g->ev[i], g->side[i]);
        cudaStreamWaitEvent(s, g->ev[i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &graph);
    for (int i = 0; i < n; i++)
        if (saved[i]) ctxs[i]->stream = saved[i], ctxs[i]->timer.on = timing[i];
    if (rc || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        hfem_graph_destroy(g);
        return rc ? rc : fail(c, HFEM_E_CUDA, "graph capture: %s", cudaGetErrorString(ee));
    }
    g->graph = graph;
    const cudaError_t ie = cudaGraphInstantiate(&g->exec, graph, 0);
    if (ie != cudaSuccess) {
        hfem_graph_destroy(g);
        return fail(c, HFEM_E_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
    }
    *out = g;
    return 0;
}

int hfem_graph_launch(hfem_graph* g, void* stream) {
    if (!g || !g->exec || !stream) return HFEM_E_ARG;
    return cudaGraphLaunch(g->exec, (cudaStream_t)stream) == cudaSuccess ? 0 : HFEM_E_CUDA;
}

int hfem_graph_destroy(hfem_graph* g) {
    if (!g) return HFEM_E_ARG;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    for (auto st : g->side)
        if (st) cudaStreamDestroy(st);
    for (auto e : g->ev)
        if (e) cudaEventDestroy(e);
    delete g;
    return 0;
}

int hfem_matvec(hfem_ctx* c, const double* x, double* y) {
    if (!c || !x || !y) return HFEM_E_ARG;
    if (!c->assembled) return fail(c, HFEM_E_STATE, "assemble before a matvec");
    CK(cudaSetDevice(c->device));
    int rc = matvec_warp(c, x, y, false, nullptr);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int hfem_set_step(hfem_ctx* c, const double* duh) {
    if (!c || !duh) return HFEM_E_ARG;
    if (!c->assembled) return fail(c, HFEM_E_STATE, "assemble before setting a step");
    CK(cudaSetDevice(c->device));
    int rc = ensure_krylov(c, 1);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->x, duh, sizeof(double) * nvec(c), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int hfem_get_ordering(hfem_ctx* c, int* ordered2unordered) {
    if (!c || !ordered2unordered) return HFEM_E_ARG;
    if (!c->have_order) return fail(c, HFEM_E_STATE, "no ordering yet (run hfem_gmres with precond 0)");
    std::memcpy(ordered2unordered, c->h_o2u.data(), sizeof(int) * c->h_o2u.size());
    return 0;
}

int hfem_reset_ordering(hfem_ctx* c) {
    if (!c) return HFEM_E_ARG;
    c->have_order = false;
    return 0;
}

int hfem_pool_trim(void) { return (int)pool_trim_device(-1); }

long long hfem_pool_cached_bytes(void) {
    std::lock_guard<std::mutex> g(pool().m);
    return (long long)pool().cached;
}

int hfem_set_precision(hfem_ctx* c, int mode) {
    if (!c) return HFEM_E_ARG;
    if (mode < 0 || mode > 3)
        return fail(c, HFEM_E_ARG, "precision mode must be 0 (FP64), 1 (3xTF32 element contractions, TF32 Schur, "
                                   "FP32 preconditioner), 2 (FP32 preconditioner) or 3 (3xTF32 element "
                                   "contractions, FP32 preconditioner)");
    c->precision = mode;
    c->assembled = false;
    return 0;
}

int hfem_gmres_problems(hfem_ctx* c, int precond, int restart, double tol, int maxit, int* conv, int* iters) {
    if (!c) return HFEM_E_ARG;
    return gmres_seg_impl(c, precond, restart, tol, maxit, conv, iters);
}

int device_buffer(hfem_ctx* c, int what, const double** src, size_t* need) {
    const hfem_dims& d = c->dims;
    switch (what) {
        case 0: *src = c->Hg; *need = (size_t)d.nblocks * c->bsz * c->bsz; break;
        case 1: *src = c->Rg; *need = (size_t)d.nf * c->bsz; break;
        case 2: *src = c->Rr; *need = (size_t)d.nf * c->bsz; break;
        case 3: *src = c->DinvRu; *need = (size_t)d.ne * c->n; break;
        case 4: *src = c->DinvF; *need = (size_t)d.ne * c->n * c->nb; break;
        case 5: *src = c->H; *need = (size_t)d.ne * c->nb * c->nb; break;
        case 6: *src = c->Rh; *need = (size_t)d.ne * c->nb; break;
        case 7: *src = c->x; *need = (size_t)d.nf * c->bsz; break;
        case 8: *src = c->udg; *need = (size_t)d.ne * d.npv * c->nc; break;
        case 9: *src = c->uh; *need = (size_t)d.nf * d.npf * c->nch; break;
        case 10: *src = c->K; *need = (size_t)d.ne * c->nb * c->n; break;
        case 12: *src = c->Ro; *need = (size_t)d.ne * c->nb; break;
        case 13: *src = c->D; *need = (size_t)d.ne * c->n * c->n; break;
        case 14: *src = c->ru2; *need = (size_t)d.ne; break;
        default: return fail(c, HFEM_E_ARG, "unknown buffer %d", what);
    }
    if (!*src) return fail(c, HFEM_E_STATE, "nothing computed for buffer %d yet", what);
    return 0;
}

int hfem_device_buffer(hfem_ctx* c, int what, const double** ptr, size_t* count) {
    if (!c || !ptr || !count) return HFEM_E_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return device_buffer(c, what, ptr, count);
}

int hfem_download(hfem_ctx* c, int what, double* host, size_t count) {
    if (!c || !host) return HFEM_E_ARG;
    const double* src = nullptr;
    size_t need = 0;
    int rc = device_buffer(c, what, &src, &need);
    if (rc) return rc;
    if (count < need) return fail(c, HFEM_E_ARG, "buffer of %zu < %zu entries", count, need);
    CK(cudaMemcpyAsync(host, src, sizeof(double) * need, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return 0;
}

int hfem_set_timing(hfem_ctx* c, int on) {
    if (!c) return HFEM_E_ARG;
    flush_timer(c);
    c->timer.on = on != 0;
    c->timer.acc.clear();
    return 0;
}

int hfem_kernel_times(hfem_ctx* c, char* names, size_t names_len, double* ms, int* counts, int max_kernels) {
    if (!c || !names || !ms) return HFEM_E_ARG;
    flush_timer(c);
    std::string s;
    int i = 0;
    for (auto& kv : c->timer.acc) {
        if (i >= max_kernels) break;
        if (i) s += ";";
        s += kv.first;
        ms[i] = kv.second.first;
        if (counts) counts[i] = kv.second.second;
        i++;
    }
    if (s.size() + 1 > names_len) return fail(c, HFEM_E_ARG, "names buffer too small");
    std::memcpy(names, s.c_str(), s.size() + 1);
    return i;
}

// FP64 FMA burst: the compute roof of the FP64 element path on this device.
__global__ void fp64_burst_kernel(int iters, double seed, double* out) {
    double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
           a7 = a0 + 7;
    const double b = 0.999999, c = 1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
            a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678) out[0] = s;
}

int hfem_fp64_peak(int device, double* tflops) {
    if (!tflops) return HFEM_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return HFEM_E_CUDA;
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double)) != cudaSuccess) return HFEM_E_NOMEM;
    const int blocks = sms(device) * 8, threads = 256, iters = 2048;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 0.0;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(a);
        fp64_burst_kernel<<<blocks, threads>>>(iters, 1.0 + r, d);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        if (r > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(d);
    if (cudaGetLastError() != cudaSuccess) return HFEM_E_CUDA;
    *tflops = best;
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Element assembly + condensation with no device allocation.
//
// For callers that hand out all device memory themselves and must not call
// cudaMalloc: programs whose memory comes from a caching pool (a PyTorch or
// RMM allocator, where a raw cudaMalloc synchronises the device and fragments
// the pool), serving loops that reserve HBM once at admission and may not
// allocate per request, and host codes that register a fixed set of buffers.
// It runs the kernels of hfem_assemble (element_kernel, the blocked
// Gauss-Jordan inverse, the fused condensation and Rh - K D^-1 Ru), so its
// blocks equal that path's; only the element kernel's per-CTA workspace lives
// in the file-scope array below instead of a context buffer.  The array's size
// is fixed at HFEM_NOALLOC_SCRATCH_BYTES (32 MiB) on every GPU that loads this
// library, for the life of the process; it caps the element kernel's grid at
// the number of workspace slots that fit (fewer CTAs for large element shapes,
// same results).
// ---------------------------------------------------------------------------
#define HFEM_NOALLOC_SCRATCH_BYTES (32u << 20)
static __device__ __align__(256) double g_noalloc_scratch[HFEM_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kMaxDevices] = {nullptr};
// per (device, element shape): attributes set and grid sizes computed once
struct NoallocGrids {
    bool ready = false;
    int elem = 0, inv = 0;
};
NoallocGrids g_noalloc_grids[kMaxDevices][16];
}  // namespace

extern "C" int hfem_condense_noalloc(const hfem_dims* dims, const double* shapvt, const double* shapvg,
                                     const double* shapvgdotshapvl, const double* shapft, const double* shapfg,
                                     const double* shapfgdotshapfc, const int* perm, const double* dgnodes,
                                     const int* elcon, const double* udg, const double* uh, const double* sh,
                                     const double* physicsparam, int tdep, double fc_u, double fc_q, const int* bf,
                                     const int* bcm, const double* bcs, int appname, double* D, double* DinvF,
                                     double* K, double* H, double* DinvRu, double* Rh, double* Rh_uncondensed,
                                     double* ru2, int* info, void* stream) {
    if (!dims || !shapvt || !shapvg || !shapvgdotshapvl || !shapft || !shapfg || !shapfgdotshapfc || !perm ||
        !dgnodes || !elcon || !udg || !uh || !sh || !physicsparam || !D || !DinvF || !K || !H || !DinvRu || !Rh ||
        !Rh_uncondensed || !ru2 || !info || (bf && (!bcm || !bcs)) || (appname != 0 && appname != 1))
        return HFEM_E_ARG;
    const hfem_dims& d = *dims;
    if (d.ne <= 0) return HFEM_E_ARG;
    int li = -1;
    const std::vector<Launch>& all = launches();
    for (size_t k = 0; k < all.size(); k++)
        if (all[k].nd == d.nd && all[k].npv == d.npv && all[k].npf == d.npf && all[k].ngv == d.ngv &&
            all[k].ngf == d.ngf)
            li = (int)k;
    if (li < 0) return HFEM_E_UNSUPPORTED;
    const Launch* L = &all[li];
    const size_t slot_bytes = L->ws * sizeof(double);
    if (slot_bytes > HFEM_NOALLOC_SCRATCH_BYTES) return HFEM_E_ARG;   // one CTA's workspace exceeds the scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HFEM_E_CUDA;
    double* scratch = nullptr;
    int ge = 0, gi = 0;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            // once per device, with that device current
            if (cudaGetSymbolAddress((void**)&g_noalloc_ptr[dev], g_noalloc_scratch) != cudaSuccess) {
                g_noalloc_ptr[dev] = nullptr;
                return HFEM_E_CUDA;
            }
        }
        scratch = g_noalloc_ptr[dev];
        NoallocGrids& G = g_noalloc_grids[dev][li];
        if (!G.ready) {
            if (cudaFuncSetAttribute(L->elem_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->elem_smem) !=
                    cudaSuccess ||
                cudaFuncSetAttribute(L->inv_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->inv_smem) !=
                    cudaSuccess ||
                cudaFuncSetAttribute(L->fused_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->fused_smem) !=
                    cudaSuccess)
                return HFEM_E_CUDA;
            int occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L->elem_fn, NT, L->elem_smem);
            const int slots = (int)(HFEM_NOALLOC_SCRATCH_BYTES / slot_bytes);
            G.elem = std::max(1, std::min(slots, sms(dev) * std::max(occ, 1)));
            occ = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, L->inv_fn, L->inv_threads, L->inv_smem);
            G.inv = sms(dev) * std::max(occ, 1);
            G.ready = true;
        }
        ge = std::min(d.ne, G.elem);
        gi = std::min(d.ne, G.inv);
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int n = L->npv * (d.nd + 2), nb = (d.nd + 2) * d.npf * (d.nd + 1);

    ElemArgs a;
    a.T = Tables{shapvt, shapvg, shapvgdotshapvl, shapft, shapfg, shapfgdotshapfc, perm};
    a.dgnodes = dgnodes;
    a.elcon = elcon;
    a.udg = udg;
    a.uh = uh;
    a.sh = sh;
    for (int i = 0; i < 6; i++) a.param[i] = physicsparam[i];
    a.tdep = tdep;
    a.fc_u = fc_u;
    a.fc_q = fc_q;
    a.ne = d.ne;
    // F is formed in the DinvF buffer and condensed there in place
    a.D = D; a.F = DinvF; a.K = K; a.H = H;
    a.Ru = DinvRu; a.Rh = Rh; a.Ro = Rh_uncondensed; a.ru2 = ru2;
    a.ws = scratch;
    a.eprob = nullptr;
    a.pparam = nullptr;
    a.bf = bf;
    a.bcm = bcm;
    a.bcs = bcs;
    a.inviscid = appname == 0;
    L->element(dim3(ge), L->elem_smem, st, a);
    if (cudaGetLastError() != cudaSuccess) return HFEM_E_CUDA;
    L->inverse(dim3(gi), st, d.ne, D, DinvRu, DinvRu, info);
    if (cudaGetLastError() != cudaSuccess) return HFEM_E_CUDA;
    LiftArgs lh;
    lh.src = H;
    lh.perm = perm;
    lh.bf = bf;
    lh.npv = d.npv;
    lh.npf = d.npf;
    lh.nfe = d.nfe;
    lh.nch = d.nd + 2;
    lh.cols = nb;
    // F (formed in the DinvF buffer) += P H, then the condensation in place
    lift_inplace_kernel<<<sms(dev) * 8, 32 * LIFT_WARPS, 0, st>>>(d.ne, n, lh, DinvF);
    if (cudaGetLastError() != cudaSuccess) return HFEM_E_CUDA;
    L->schur_fused(st, d.ne, D, DinvF, K, H, DinvF);
    if (cudaGetLastError() != cudaSuccess) return HFEM_E_CUDA;
    batched_dgemv_kernel<<<sms(dev) * 8, 256, 0, st>>>(d.ne, nb, n, -1.0, K, (long long)nb * n, DinvRu, n, Rh, nb);
    if (cudaGetLastError() != cudaSuccess) return HFEM_E_CUDA;
    return 0;
}
