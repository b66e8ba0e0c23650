// Internal declarations shared by the CUDA translation units of libtgap.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "../../include/tgap.h"

namespace tgap {

// Compile-time bounds of the descriptor kernels.
constexpr int kMaxSpecies = 4;
constexpr int kMaxAlpha = 16;     // radial functions per species
constexpr int kMaxNmax = 16;      // radial functions summed over species
constexpr int kMaxL = 10;         // l_max
constexpr int kMaxNodes = 192;    // quadrature nodes per species
// Radial table intervals over [0, rcut_hard] (mixed path). The cubic Hermite interpolant's error
// against the FP64 radial functions is 6.6e-9 of max |R_n| at 256 intervals for the carbon
// settings (rcut 3.7 A, sigma 0.5 A; 2.5e-11 at 1024, 1.0e-7 at 128), ten times below the FP32
// rounding of the stored coefficients, and the table (32 KB per species at alpha_max 8) stays in L1.
constexpr int kTabIntervals = 256;

struct Error {
    int status;
    std::string msg;
};

// Incremented by every device (re)allocation or release of a DevBuf; a captured CUDA graph is
// valid only while the epoch it was captured at is current.
extern std::atomic<uint64_t> g_alloc_epoch;

// Growable device buffer owned by a context or object.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int ensure(size_t n);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Pinned host staging buffer.
struct HostBuf {
    void *ptr = nullptr;
    void *dev = nullptr;  // its address in the device's address space (pinned memory is mapped)
    size_t bytes = 0;
    int ensure(size_t n);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

}  // namespace tgap

namespace tgap {
struct StageRecord {
    int stage;
    cudaEvent_t start, stop;
};
}  // namespace tgap

struct tgap_context {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int64_t launches = 0;
    // scratch buffers reused across calls (host-buffer entry points)
    tgap::DevBuf scratch[24];
    tgap::HostBuf pinned[4];
    // caller arrays page-locked (and mapped) with tgap_host_register
    struct HostRegion {
        uintptr_t host;
        size_t bytes;
        uintptr_t dev;  // its address in the device's address space
    };
    std::vector<HostRegion> registered;
    int *d_flag = nullptr;  // device error flag (bounded waits, overflow)
    int *d_check = nullptr; // device check word: code, index, value, failures (int[4])
    bool sync_check = false;  // TGAP_SYNC_CHECK=1: synchronize and read the check after each launch
    // stage timing
    bool timing = false;
    std::vector<std::string> stage_names;
    std::vector<double> stage_ms;
    std::vector<int64_t> stage_count;
    std::vector<tgap::StageRecord> pending;
    std::vector<cudaEvent_t> event_pool;
    // autotuned launch choices (tgap_autotune): key -> value. Launchers register their key, the
    // stage that times it and the candidate values on first use; while tuning, probe_key's value
    // is forced to probe_val.
    struct TuneSlot {
        std::string stage;
        std::vector<int> candidates;
        int dflt = 0;
    };
    std::map<std::string, int> tune;
    std::vector<std::pair<std::string, int>> tune_suffix;  // tgap_autotune_set("*suffix", v)
    std::map<std::string, TuneSlot> tune_seen;
    std::string probe_key;
    int probe_val = 0;
    std::string tune_report;
};

namespace tgap {

// Brackets one kernel stage with CUDA events on the context stream when timing is enabled.
class StageScope {
  public:
    StageScope(tgap_context *ctx, const char *name);
    ~StageScope();

  private:
    tgap_context *ctx_;
    int rec_ = -1;
};

int set_error(tgap_context *ctx, int status, const char *fmt, ...);
// Error message of an entry point that has no context (per host thread; tgap_last_error(NULL)).
int thread_error(int status, const char *fmt, ...);

// Launch choice for `key`: the probed value while the autotuner times it, else the tuned value,
// else dflt. Registers the key with its timing stage and candidates (the first candidate list
// seen for a key is kept).
int tuned(tgap_context *ctx, const std::string &key, const char *stage, const std::vector<int> &candidates, int dflt);
int cuda_check(tgap_context *ctx, cudaError_t e, const char *what);

#define TGAP_CUDA(ctx, call)                                           \
    do {                                                               \
        cudaError_t _e = (call);                                       \
        if (_e != cudaSuccess) return ::tgap::cuda_check(ctx, _e, #call); \
    } while (0)

// Reads and clears the device check word; a recorded failure becomes TGAP_ERR_NUMERIC (code
// kCheckNonFinite) or TGAP_ERR_CUDA (an index out of bounds). Synchronizes the context stream.
int read_device_check(tgap_context *ctx);
// With ctx->sync_check set and the stream not capturing: synchronize and read the check word.
int sync_check_launch(tgap_context *ctx);

#define TGAP_LAUNCH_CHECK(ctx)                                         \
    do {                                                               \
        (ctx)->launches++;                                             \
        cudaError_t _e = cudaGetLastError();                           \
        if (_e != cudaSuccess) return ::tgap::cuda_check(ctx, _e, "kernel launch"); \
        if ((ctx)->sync_check) {                                       \
            int _rc = ::tgap::sync_check_launch(ctx);                  \
            if (_rc) return _rc;                                       \
        }                                                              \
    } while (0)

// Codes of the device check word.
enum CheckCode {
    kCheckNone = 0,
    kCheckFwdPair = 1,      // descriptor forward: compacted pair outside its site (not raised since
                            // the compaction stages only the site's own pairs; the code stays reserved)
    kCheckBwdPair = 2,      // adjoint: the same (reserved)
    kCheckBwdAtom = 3,      // adjoint: neighbor atom index out of range
    kCheckSelfAtom = 4,     // adjoint: self-slot atom index out of range
    kCheckNonFinite = 5,    // velocity Verlet: non-finite force
    kCheckListOverrun = 6,  // neighbor fill wrote past its counted range
    kCheckMcOverflow = 7,   // Monte Carlo: affected sites or pairs beyond the trial capacity
    kCheckPairCapacity = 8, // device-side list rebuild: more pairs than the reserved capacity
};

#ifdef __CUDACC__
// Programmatic dependent launch, at the top of a kernel launched with launch_pdl: wait until the
// preceding kernel's grid has completed and its memory is visible, then allow the next kernel to
// be scheduled (it holds at its own wait until this grid completes). Outside such a launch both
// instructions do nothing.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches kern with programmatic stream serialization: its blocks may be scheduled while the
// preceding kernel finishes; kern must call pdl_enter() before reading that kernel's output.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                              Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

// Records the first failure (code, index, value) and counts all of them; the access that failed
// is skipped by the caller.
__device__ __forceinline__ void check_fail(int *check, int code, long long index, long long value)
{
    if (!check) return;
    if (atomicCAS(check, 0, code) == 0) {
        check[1] = (int)index;
        check[2] = (int)value;
    }
    atomicAdd(check + 3, 1);
}
#endif

// ---------------------------------------------------------------------------- hypers

// Descriptor settings in device-friendly form (one per model), plus host-built tables.
struct SoapParams {
    int n_species;
    int l_max;
    int n_max;              // sum of alpha_max
    int dim;                // n_max (n_max + 1) / 2 (l_max + 1)
    int radial_enhancement;
    int alpha_max[kMaxSpecies];
    int n_off[kMaxSpecies];  // first radial index of each species block
    int n_nodes[kMaxSpecies];
    int node_off[kMaxSpecies];
    int tq_off[kMaxSpecies];
    int max_alpha;
    int am_pad;              // max_alpha rounded up to 4 (radial table row length)
    double tab_scale[kMaxSpecies];  // kTabIntervals / rcut_hard
    double rcut_hard[kMaxSpecies], rcut_soft[kMaxSpecies], nf[kMaxSpecies];
    double global_scaling[kMaxSpecies], sigma_r[kMaxSpecies], sigma_r_scaling[kMaxSpecies];
    double sigma_t[kMaxSpecies], sigma_t_scaling[kMaxSpecies];
    double amplitude_scaling[kMaxSpecies], central_weight[kMaxSpecies];
    double rcut_max;
    // SOAP compression (read_gap.f90:489-559): q = P p / |P p|, P sparse (dim_out x dim); without it
    // dim_out = dim and the pointers are null. P by rows (output components, for the forward) and by
    // columns (power-spectrum components, for the adjoint's P^T), each in the order given.
    int dim_out;
    const int *cmp_row, *cmp_rcol;  // row offsets [dim_out + 1], column of each entry
    const int *cmp_col, *cmp_crow;  // column offsets [dim + 1], row of each entry
    const double *cmp_rval, *cmp_cval;
    const float *cmp_rval32, *cmp_cval32;
};

// Host-side tables: quadrature node positions, weighted orthonormal basis values
// (node-major, alpha_max per node) and the central-atom radial coefficients.
struct SoapTables {
    std::vector<double> xq;       // sum n_nodes
    std::vector<double> tq;       // sum n_nodes * alpha_max
    std::vector<double> central;  // n_max (R_n(0) * central_weight * Y_00 per species block)
};

int make_soap_params(const tgap_soap_hypers *h, SoapParams *p, std::string *why);
// tables.cpp (binary128 arithmetic on the host)
int build_soap_tables(const SoapParams &p, SoapTables *t);
void poly3_orthonormaliser(int alpha_max, double *W);  // W = S^{-1/2}, row-major

// Device copy of the tables for one model.
struct DeviceSoap {
    SoapParams p;
    DevBuf xq, tq, central;
    float *xq_f = nullptr, *tq_f = nullptr, *central_f = nullptr;  // single-precision copies
    DevBuf xq32, tq32, central32;
    DevBuf rtab;  // float4 [n_species][kTabIntervals][am_pad]: cubic Hermite radial table
    DevBuf cmp_i, cmp_f64, cmp_f32;  // compression: offsets and indices (int), values (FP64, FP32)
};
int upload_soap(tgap_context *ctx, const SoapParams &p, const SoapTables &t, DeviceSoap *d);

// ---------------------------------------------------------------------------- pairs

// Read-only view of a neighbor list for the descriptor kernels.
// Descriptor forward only: with pos set, each site's warp first writes the minimum-image pair
// vectors and distances of its list pairs (rjs_out / xyz_out, the arrays the view reads) from the
// primitive positions, so a per-step geometry pass is not needed. sd: const StructDesc *.
struct GeomSrc {
    const double *pos = nullptr;
    const int *list = nullptr;
    const int *site_struct = nullptr;
    const void *sd = nullptr;
    double *rjs_out = nullptr;
    double *xyz_out = nullptr;
};

struct PairView {
    const int64_t *start;   // [n_sites_total + 1]
    const double *xyz;      // [3 P]  r_j - r_i (minimum image)
    const double *rjs;      // [P]
    const int *species;     // [P]    species channel of the neighbor (1-based, 0 = blind)
    const int *jatom;       // [P]    folded global neighbor index (force scatter)
    int n_atoms;            // bound of jatom
    int *check;             // device check word
    // adjoint only: when set, dq_i/dr_j contracted with dE_i/dq_i is written per pair (3 per list
    // pair, self slot = minus the sum) instead of being scattered into forces and virial
    double *pair_der = nullptr;
    const double *gate = nullptr;  // with pair_der: sites whose gate value is 0 write nothing
    GeomSrc geo;                   // descriptor forward: pair geometry from positions
    // persistent form: a zeroed site counter the launch's warps take sites from (grid sized to
    // what is resident at once); null: one site per warp
    int *queue = nullptr;
};

// Site counters of one evaluation (two per model: forward, adjoint), zeroed with its outputs.
constexpr int kQueueInts = 64;

}  // namespace tgap
