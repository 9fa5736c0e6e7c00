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
        float us[4];
    };
    std::map<std::vector<int>, TuneEntry> tune;
    c2q::SolverScalars* tune_scratch = nullptr;  // reductions of tuning launches land here
    bool autotune = true;
    int sm_count  = 0;
    // pinned ring of the batched solvers: 4 slots x 16 right-hand sides x 4 doubles
    double* batch_ring = nullptr;
};

struct c2q_gauge {
    c2q_ctx* ctx = nullptr;
    c2q_lattice lat{};
    c2q::Geom geom{};
    // [0] FP64 18-real, [1] FP64 12-real, [2] FP32 18-real, [3] FP32 12-real, [4] FP16 12-real,
    // [5] FP16 18-real
    c2q::GaugeStore store[6];
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

enum GaugeKind { G64 = 0, G64R12 = 1, G32 = 2, G32R12 = 3, G16R12 = 4, G16 = 5 };

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
int ensure_staging(c2q_ctx* ctx, size_t bytes);
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
    int dot = 0;
    int fin = FIN_STORE_RESULT;
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
