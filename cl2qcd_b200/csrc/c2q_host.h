// c2q_host.h -- host-side objects behind the C ABI: context (stream, reduction
// scratch, device scalars), gauge fields in every storage precision, eo spinor
// fields, and the launch wrappers the solvers are built from.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/cl2qcd_b200.h"
#include "c2q_internal.cuh"
#include "blas.cuh"
#include "pack.cuh"
#include "reduce.cuh"

namespace c2q {

struct Field;

// Storage of one gauge field in one precision / compression.
struct GaugeStore {
    void* data = nullptr;
    size_t bytes = 0;
};

}  // namespace c2q

struct c2q_ctx {
    int device        = 0;
    cudaStream_t stream = nullptr;
    bool own_stream   = false;
    std::string err;
    long long launches = 0;
    // reduction scratch (partials), the last-block ticket and result slots
    double* partials       = nullptr;
    size_t partials_cap    = 0;  // doubles
    unsigned* ticket       = nullptr;
    double* red_result     = nullptr;  // 8 doubles
    double* host_pinned    = nullptr;  // 64 doubles, pinned
    c2q::SolverScalars* scalars = nullptr;  // device solver scalars (one set per context)
    // staging buffer for AoS host <-> device transfers
    void* staging          = nullptr;
    size_t staging_cap     = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ring_ev[4] = {};  // residual ring of the pipelined solvers
    // The pipelined solvers copy each iteration's residual into ring_dev on the
    // context's stream (device memory only) and forward it to pinned host memory
    // on `monitor`, so the solve never waits on a write across PCIe, which a large
    // transfer of another stream can hold up; ring_ev[k] completes when slot k
    // has reached the host, mon_ev[k] when it is in ring_dev.
    cudaStream_t monitor   = nullptr;
    cudaEvent_t mon_ev[4]  = {};
    double* ring_dev       = nullptr;  // 4 slots x 16 right-hand sides x 4 doubles
    // optional per-launch dslash timing (c2q_ctx_profile)
    bool profiling = false;
    struct Timed {
        cudaEvent_t a, b;
        int prec;
        double sites;
        double bytes;  // algorithmic bytes of the launch
    };
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> event_pool;
    // link storage of the explicit operator entry points: 0 18-real, 1 12-real
    int rec12 = 0;
    // autotuner of the paired-site dslash: launch shape -> chosen configuration
    struct TuneEntry {
        int cfg;
        float us[5];  // per choice; 0 where a choice does not apply to the shape
    };
    std::map<std::vector<int>, TuneEntry> tune;
    c2q::SolverScalars* tune_scratch = nullptr;  // reductions of tuning launches land here
    bool autotune = true;
    // dependent launches of the solver-loop kernels (launch_dep); environment
    // C2Q_DEPENDENT_LAUNCH=0 turns them off for new contexts
    bool pdl = true;
    int force_choice = -1;  // >= 0: every paired-site sweep uses this choice where it applies
    // launch predicate of a device-driven solve (SolverScalars::halt): while set,
    // every reducing BLAS and dslash launch skips its work once *halt_dev != 0
    const int* halt_dev = nullptr;
    int sm_count  = 0;
    // pinned ring of the batched solvers: 4 slots x 16 right-hand sides x 4 doubles
    double* batch_ring = nullptr;
    // device aliases of the pinned host buffers above (small solver transfers are
    // copied by a one-block kernel through them, keeping them off the copy engines,
    // where a large transfer of another stream would hold them up)
    double* host_pinned_dev = nullptr;
    double* batch_ring_dev  = nullptr;
};

struct c2q_gauge {
    c2q_ctx* ctx = nullptr;
    c2q_lattice lat{};
    c2q::Geom geom{};
    // [0] FP64 18-real, [1] FP64 12-real, [2] FP32 18-real, [3] FP32 12-real, [4] FP16 12-real,
    // [5] FP16 18-real; [6..9] the FP32 / FP16 kinds of the field in the temporal gauge
    c2q::GaugeStore store[10];
    // temporal gauge: the transformation G(x) (FP64, [parity][9 lanes][stride])
    // and the weight of the T hop leaving the last time slice
    c2q::GaugeStore tg_transform;
    double tg_lam_re = 1.0, tg_lam_im = 0.0;
    // max |row 2 - conj(row0 x row1)| of the uploaded links (-1: not measured yet)
    double rec12_dev = -1.0;
};

struct c2q_spinor_eo {
    c2q_ctx* ctx = nullptr;
    c2q_lattice lat{};
    c2q::Geom geom{};
    int prec   = 64;
    void* data = nullptr;
    float* norm = nullptr;  // FP16 only
    bool owned = true;
};

namespace c2q {

enum GaugeKind {
    G64 = 0, G64R12 = 1, G32 = 2, G32R12 = 3, G16R12 = 4, G16 = 5,
    G32TG = 6, G32R12TG = 7, G16R12TG = 8, G16TG = 9,  // the same in the temporal gauge
    GAUGE_KINDS = 10
};
inline bool gkind_is_tg(int k) { return k >= G32TG && k <= G16TG; }
inline bool gkind_is_r12(int k) { return k == G64R12 || k == G32R12 || k == G16R12 || k == G32R12TG || k == G16R12TG; }
// the temporal-gauge kind of a FP32 / FP16 kind
inline int gkind_tg(int k)
{
    return k == G32 ? G32TG : k == G32R12 ? G32R12TG : k == G16R12 ? G16R12TG : k == G16 ? G16TG : -1;
}

// ---- status plumbing ----
int fail(c2q_ctx* ctx, int code, const std::string& msg);
int cuda_fail(c2q_ctx* ctx, cudaError_t e, const char* where);
#define C2Q_CUDA(ctx, call)                                   \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return ::c2q::cuda_fail((ctx), _e, #call); \
    } while (0)

// ---- geometry / coefficients ----
bool make_geom(const c2q_lattice& lat, Geom* g);
bool same_lattice(const c2q_lattice& a, const c2q_lattice& b);
// A constant as the reference passes it in its build options (16 significant digits).
double as_build_option(double v);
// Hop coefficients for one launch: -kappa * boundary phase (and chemical potential on T).
HopCoef hop_coef(const c2q_lattice& lat, double kappa);
EpiArgs diag_epi(double mubar, int which, int gamma5);

// gauge storage for operator sweeps at precision `prec` (FP16 links are always 12-real)
int gkind_for(int prec, int rec12);

// ---- fields ----
// Allocate a spinor field of storage precision `prec` (stream-ordered allocation).
int field_alloc(c2q_ctx* ctx, const c2q_lattice& lat, int prec, c2q_spinor_eo* f);
void field_free(c2q_spinor_eo* f);
size_t field_bytes(const Geom& g, int prec);
int gauge_ensure(c2q_gauge* g, int kind);  // builds a lower-precision copy on first use
// frees every copy derived from the FP64 18-real links (rebuilt on next use)
int gauge_drop_derived(c2q_gauge* g);
// 12-real FP64 links are the same operator as the uploaded 18-real ones when
// row 2 of every link equals conj(row0 x row1) to this tolerance (unitarity.cu)
constexpr double REC12_EXACT_TOL = 1e-13;
bool rec12_exact(c2q_gauge* g);
// the FP64 links a solver's residuals use: 12-real only where they are the same operator
inline int gk64_for(const c2q_gauge* g, int rec12)
{
    return rec12 && rec12_exact(const_cast<c2q_gauge*>(g)) ? G64R12 : G64;
}

// ---- temporal gauge (tgauge.cu) ----
// The inner solves of the mixed-precision CG may run on the field transformed
// by G(x, t) = c^t prod_{t' < t} U_T(x, t') (c the forward T phase): every T
// link becomes the identity except the one leaving the last time slice, which
// becomes lambda W (W in SU(3), lambda = c^NT), all hop phases real.  Possible
// when the T weights are pure phases and the spatial ones real.
bool tg_applicable(const c2q_lattice& lat);
// the transformation G and lambda (first use)
int tg_ensure(c2q_gauge* g);
// the transformed links as an FP64 9-lane store (the layout of G64) in out
int tg_links_fp64(c2q_gauge* g, void* out);
// out (FP32) = G in (FP64), on the sites of parity 1 (those of the CG vectors)
int tg_to_inner(c2q_ctx* ctx, const c2q_gauge* g, c2q_spinor_eo* out, const c2q_spinor_eo* in);
// x (FP64) += G^dagger (xs + alpha p) (alpha from sc; sc null: xs only), xs = 0
int tg_accumulate(c2q_ctx* ctx, const c2q_gauge* g, c2q_spinor_eo* x, c2q_spinor_eo* xs, const c2q_spinor_eo* p,
                  const SolverScalars* sc);
int ensure_staging(c2q_ctx* ctx, size_t bytes);
// Small copies (multiples of 4 bytes) between device memory and the device alias
// of a pinned host buffer, by a one-block kernel on the context's stream:
// `height` rows of `width` bytes, rows `dpitch` / `spitch` bytes apart.
int pinned_copy(c2q_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                int height = 1, cudaStream_t stream = nullptr);
// Residual ring slot k (n rows of `width` bytes at src, row pitch spitch): into
// ring_dev on the context's stream, then to the pinned host buffer dst_host_dev
// (the device alias of a pinned slot) on the monitor stream; ring_ev[k % 4]
// completes when the host can read it.
int ring_push(c2q_ctx* ctx, int k, double* dst_host_dev, const void* src, size_t spitch, size_t width, int n);
int ensure_partials(c2q_ctx* ctx, size_t blocks);

template <int P>
inline SpinorPtr<P> sptr(const c2q_spinor_eo* f)
{
    return SpinorPtr<P>{f ? f->data : nullptr, f ? f->norm : nullptr, f ? f->geom.seo / 2 : 0};
}

// ---- launches (all stream-ordered on ctx->stream) ----
struct DotSpec {
    int mode = 0;  // DotMode
    const c2q_spinor_eo* y = nullptr;
    int fin = FIN_STORE_RESULT;
};

// One dslash parity sweep at the fields' storage precision P.
int launch_dslash(c2q_ctx* ctx, const c2q_gauge* g, int gkind, c2q_spinor_eo* out, const c2q_spinor_eo* in,
                  int out_parity, double kappa, int epi, const EpiArgs& e, const c2q_spinor_eo* x,
                  const DotSpec& dot);
struct BlasSpec {
    int op = 0;
    Coef a{0, 0, nullptr, 1}, b{0, 0, nullptr, 1};
    c2q_spinor_eo* out = nullptr;
    const c2q_spinor_eo *x = nullptr, *y = nullptr, *z = nullptr;
    const c2q_spinor_eo* w = nullptr;  // B_BICG_XR
    c2q_spinor_eo* out2    = nullptr;  // B_BICG_XR
    int dot = 0;
    int fin = FIN_STORE_RESULT;
    int fin_arg = 0;
};
int launch_blas(c2q_ctx* ctx, const BlasSpec& s);
int launch_cg_update(c2q_ctx* ctx, c2q_spinor_eo* x, c2q_spinor_eo* r, const c2q_spinor_eo* p,
                     const c2q_spinor_eo* v);
int launch_cg_p(c2q_ctx* ctx, c2q_spinor_eo* p, const c2q_spinor_eo* r);
int launch_convert(c2q_ctx* ctx, c2q_spinor_eo* out, const c2q_spinor_eo* in);

// A batch of right-hand sides for one sweep of the paired-site dslash
// (FP32 / FP16 fields, pdslash.cuh): per right-hand side r, out[r] = epilogue
// of the hopping term on in[r], with x[r] the EPI_AXPY operand, y[r] the DOT_Y
// partner and sc[r] the solver scalars its reduction finishes into.
constexpr int MAX_BATCH = PK_MAX_RHS;
struct PkBatch {
    int n = 0;
    c2q_spinor_eo* out[MAX_BATCH] = {};
    const c2q_spinor_eo* in[MAX_BATCH] = {};
    const c2q_spinor_eo* x[MAX_BATCH] = {};
    const c2q_spinor_eo* y[MAX_BATCH] = {};
    SolverScalars* sc[MAX_BATCH] = {};
    int out_parity = 0;
    double kappa = 0;
    int epi = 0;
    EpiArgs e{1, 0, 1, 0, 0};
    int dot_mode = 0;
    int fin = FIN_STORE_RESULT;
};
int launch_pdslash(c2q_ctx* ctx, const c2q_gauge* g, int gkind, const PkBatch& B);
// Batched fermion matrix on reduced-precision fields: out[r] = A in[r] for
// r < n, tmp1/tmp2 per right-hand side; optionally reduces <y[r], out[r]>
// into sc[r] with finisher `fin` (for QplusQminus_eo with y = in, as
// |Qminus_eo in|^2, which equals it because Qplus_eo = Qminus_eo^dagger).
// With r_update (QplusQminus_eo, y = in) the last sweep instead applies the CG
// residual update r[r] -= alpha A in[r] and reduces |r|^2 into sc[r] (FIN_CG_BETA);
// out[r] is then not written; with x_update as well, the third sweep applies the
// CG solution update x_update[r] += alpha in[r] (FP32 x_update).
int apply_operator_batch(c2q_ctx* ctx, int op, int n, c2q_spinor_eo* const* out, const c2q_gauge* g, int gkind,
                         const c2q_spinor_eo* const* in, double kappa, double mubar, int action,
                         c2q_spinor_eo* const* tmp1, c2q_spinor_eo* const* tmp2, int dot_mode,
                         const c2q_spinor_eo* const* y, int fin, SolverScalars* const* sc, int* sweeps,
                         c2q_spinor_eo* const* r_update = nullptr, c2q_spinor_eo* const* x_update = nullptr);
// an event for per-launch profiling (from the context's pool)
cudaEvent_t profile_event(c2q_ctx* ctx);

// Fermion matrix application at the fields' precision.  tmp1/tmp2 are
// scratch fields of the same precision.  `dot` applies to the last sweep.
int apply_operator(c2q_ctx* ctx, int op, c2q_spinor_eo* out, const c2q_gauge* g, int gkind,
                   const c2q_spinor_eo* in, double kappa, double mubar, int action, c2q_spinor_eo* tmp1,
                   c2q_spinor_eo* tmp2, const DotSpec& dot, int* sweeps);

// Read back `n` doubles of device memory synchronously through pinned memory.
int read_scalars(c2q_ctx* ctx, const double* dev, int n, double* host);

}  // namespace c2q
