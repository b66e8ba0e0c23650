// C ABI of libtgap (declarations and reference citations in include/tgap.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gap_kernels.h"
#include "mc_kernels.h"
#include "screen_kernels.h"
#include "md_kernels.h"
#include "neighbors.h"
#include "pair_kernels.h"
#include "soap_kernels.h"
#include "tgap_internal.h"

using namespace tgap;

// ============================================================================ utilities

namespace tgap {

std::atomic<uint64_t> g_alloc_epoch{0};

// Captured graphs (MD steps, host-buffer calls) are re-captured after any change of what they baked
// in: a buffer that moved, e0, the site range, a launch choice of the autotuner.
static void graphs_stale() { g_alloc_epoch.fetch_add(1, std::memory_order_relaxed); }

int DevBuf::ensure(size_t n)
{
    if (n <= bytes && ptr) return 0;
    // any (re)allocation can move a buffer that a captured graph still refers to
    g_alloc_epoch.fetch_add(1, std::memory_order_relaxed);
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    size_t want = n < 256 ? 256 : n;
    if (cudaMalloc(&ptr, want) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return 1;
    }
    bytes = want;
    return 0;
}

void DevBuf::release()
{
    if (ptr) g_alloc_epoch.fetch_add(1, std::memory_order_relaxed);
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

int HostBuf::ensure(size_t n)
{
    if (n <= bytes && ptr) return 0;
    // captured call graphs read and write the staging buffers through their device addresses
    g_alloc_epoch.fetch_add(1, std::memory_order_relaxed);
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    if (cudaMallocHost(&ptr, n < 256 ? 256 : n) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return 1;
    }
    if (cudaHostGetDevicePointer(&dev, ptr, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(ptr);
        ptr = dev = nullptr;
        return 1;
    }
    bytes = n < 256 ? 256 : n;
    return 0;
}

void HostBuf::release()
{
    if (ptr) g_alloc_epoch.fetch_add(1, std::memory_order_relaxed);
    if (ptr) cudaFreeHost(ptr);
    ptr = dev = nullptr;
    bytes = 0;
}

int set_error(tgap_context *ctx, int status, const char *fmt, ...)
{
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return status;
}

static thread_local std::string t_last_error;

int thread_error(int status, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return status;
}

const char *thread_error_text() { return t_last_error.c_str(); }

int tuned(tgap_context *ctx, const std::string &key, const char *stage, const std::vector<int> &candidates, int dflt)
{
    if (!ctx) return dflt;
    if (!ctx->probe_key.empty() && key == ctx->probe_key) return ctx->probe_val;
    if (!ctx->tune_seen.count(key)) ctx->tune_seen[key] = tgap_context::TuneSlot{stage, candidates, dflt};
    const auto it = ctx->tune.find(key);
    if (it != ctx->tune.end()) return it->second;
    for (const auto &pat : ctx->tune_suffix)
        if (key.size() >= pat.first.size() && key.compare(key.size() - pat.first.size(), pat.first.size(), pat.first) == 0)
            return pat.second;
    return dflt;
}

int cuda_check(tgap_context *ctx, cudaError_t e, const char *what)
{
    return set_error(ctx, e == cudaErrorMemoryAllocation ? TGAP_ERR_NOMEM : TGAP_ERR_CUDA,
                     "%s: %s", what, cudaGetErrorString(e));
}

StageScope::StageScope(tgap_context *ctx, const char *name) : ctx_(ctx)
{
    if (!ctx || !ctx->timing) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    int stage = -1;
    for (size_t i = 0; i < ctx->stage_names.size(); ++i)
        if (ctx->stage_names[i] == name) stage = (int)i;
    if (stage < 0) {
        stage = (int)ctx->stage_names.size();
        ctx->stage_names.push_back(name);
        ctx->stage_ms.push_back(0.0);
        ctx->stage_count.push_back(0);
    }
    StageRecord r;
    r.stage = stage;
    for (cudaEvent_t *e : {&r.start, &r.stop}) {
        if (!ctx->event_pool.empty()) {
            *e = ctx->event_pool.back();
            ctx->event_pool.pop_back();
        } else if (cudaEventCreate(e) != cudaSuccess) {
            return;
        }
    }
    cudaEventRecord(r.start, ctx->stream);
    rec_ = (int)ctx->pending.size();
    ctx->pending.push_back(r);
}

StageScope::~StageScope()
{
    if (rec_ >= 0) cudaEventRecord(ctx_->pending[rec_].stop, ctx_->stream);
}

}  // namespace tgap

template <class T>
static int upload(tgap_context *ctx, DevBuf &b, const T *h, size_t n)
{
    if (b.ensure(sizeof(T) * (n ? n : 1))) return set_error(ctx, TGAP_ERR_NOMEM, "device buffer");
    if (n) TGAP_CUDA(ctx, cudaMemcpyAsync(b.ptr, h, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
    return TGAP_OK;
}

template <class T>
static int download(tgap_context *ctx, T *h, const DevBuf &b, size_t n)
{
    if (n) TGAP_CUDA(ctx, cudaMemcpyAsync(h, b.ptr, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
    return TGAP_OK;
}

#define CHECK_RC(x)           \
    do {                      \
        int _rc = (x);        \
        if (_rc) return _rc;  \
    } while (0)

static int activate(tgap_context *ctx)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    TGAP_CUDA(ctx, cudaSetDevice(ctx->device));
    return TGAP_OK;
}

// ============================================================================ context

extern "C" const char *tgap_version(void) { return "tgap-b200 0.1 (sm_100a)"; }

extern "C" int tgap_create(int device, tgap_context **out)
{
    if (!out) return TGAP_ERR_ARGUMENT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return TGAP_ERR_CUDA;
    }
    if (device < 0 || device >= n) return TGAP_ERR_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return TGAP_ERR_CUDA;
    auto *ctx = new tgap_context();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return TGAP_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    if (upload_ylm_constants() != 0 || cudaMalloc(&ctx->d_check, 4 * sizeof(int)) != cudaSuccess ||
        cudaMemset(ctx->d_check, 0, 4 * sizeof(int)) != cudaSuccess) {
        if (ctx->d_check) cudaFree(ctx->d_check);
        cudaStreamDestroy(ctx->own_stream);
        delete ctx;
        return TGAP_ERR_CUDA;
    }
    const char *sc = std::getenv("TGAP_SYNC_CHECK");
    ctx->sync_check = sc && sc[0] == '1';
    *out = ctx;
    return TGAP_OK;
}

extern "C" int tgap_destroy(tgap_context *ctx)
{
    if (!ctx) return TGAP_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &b : ctx->scratch) b.release();
    for (auto &b : ctx->pinned) b.release();
    for (auto &r : ctx->registered) cudaHostUnregister(reinterpret_cast<void *>(r.host));
    for (auto &r : ctx->pending) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    if (ctx->d_flag) cudaFree(ctx->d_flag);
    if (ctx->d_check) cudaFree(ctx->d_check);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return TGAP_OK;
}

extern "C" int tgap_host_register(tgap_context *ctx, void *ptr, size_t bytes)
{
    CHECK_RC(activate(ctx));
    if (!ptr || bytes == 0) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_host_register: bad arguments");
    TGAP_CUDA(ctx, cudaHostRegister(ptr, bytes, cudaHostRegisterMapped));
    void *dev = nullptr;
    const cudaError_t e = cudaHostGetDevicePointer(&dev, ptr, 0);
    if (e != cudaSuccess) {
        cudaHostUnregister(ptr);
        return cuda_check(ctx, e, "cudaHostGetDevicePointer");
    }
    ctx->registered.push_back({reinterpret_cast<uintptr_t>(ptr), bytes, reinterpret_cast<uintptr_t>(dev)});
    return TGAP_OK;
}

extern "C" int tgap_host_unregister(tgap_context *ctx, void *ptr)
{
    CHECK_RC(activate(ctx));
    for (size_t i = 0; i < ctx->registered.size(); ++i)
        if (ctx->registered[i].host == reinterpret_cast<uintptr_t>(ptr)) {
            TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            TGAP_CUDA(ctx, cudaHostUnregister(ptr));
            ctx->registered.erase(ctx->registered.begin() + (long)i);
            graphs_stale();  // graphs that copy to or from it
            return TGAP_OK;
        }
    return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_host_unregister: not registered");
}

// The device address of [p, p + len) when it lies inside memory registered with
// tgap_host_register, else null.
static void *host_registered(const tgap_context *ctx, const void *p, size_t len)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    for (const auto &r : ctx->registered)
        if (a >= r.host && a + len <= r.host + r.bytes) return reinterpret_cast<void *>(r.dev + (a - r.host));
    return nullptr;
}

// Up to four 8-byte word arrays copied in one launch between device memory and mapped host memory
// (the caller's registered arrays or the pinned staging buffers), and up to two word arrays
// cleared: in a call graph one kernel costs less than a copy or memset node per array.
struct WordCopy {
    const unsigned long long *src[4];
    unsigned long long *dst[4];
    long long n[4];
    unsigned long long *zero[2];
    long long nz[2];
};

__global__ void k_copy_words(WordCopy c)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int a = 0; a < 4; ++a)
        for (long long i = t; i < c.n[a]; i += stride) c.dst[a][i] = c.src[a][i];
#pragma unroll
    for (int a = 0; a < 2; ++a)
        for (long long i = t; i < c.nz[a]; i += stride) c.zero[a][i] = 0ull;
}

static int copy_words(tgap_context *ctx, const WordCopy &c)
{
    long long most = 0;
    for (int a = 0; a < 4; ++a) most = std::max(most, c.n[a]);
    for (int a = 0; a < 2; ++a) most = std::max(most, c.nz[a]);
    if (most == 0) return TGAP_OK;
    const int grid = (int)std::min<long long>((most + 255) / 256, 2 * 148);
    k_copy_words<<<grid, 256, 0, ctx->stream>>>(c);
    TGAP_LAUNCH_CHECK(ctx);
    return TGAP_OK;
}


extern "C" int tgap_set_stream(tgap_context *ctx, void *stream)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return TGAP_OK;
}

namespace tgap {

int read_device_check(tgap_context *ctx)
{
    int h[4] = {0, 0, 0, 0};
    TGAP_CUDA(ctx, cudaMemcpyAsync(h, ctx->d_check, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h[0] == kCheckNone) return TGAP_OK;
    TGAP_CUDA(ctx, cudaMemsetAsync(ctx->d_check, 0, sizeof(h), ctx->stream));
    static const char *what[] = {"",
                                 "descriptor forward: pair outside its site",
                                 "descriptor adjoint: pair outside its site",
                                 "descriptor adjoint: neighbor atom out of range",
                                 "descriptor adjoint: self-slot atom out of range",
                                 "non-finite force",
                                 "neighbor fill past its counted range",
                                 "Monte Carlo trial capacity exceeded",
                                 "device-side list rebuild: more pairs than the reserved capacity"};
    const char *w = (h[0] > 0 && h[0] <= kCheckPairCapacity) ? what[h[0]] : "unknown check";
    const int status = h[0] == kCheckNonFinite ? TGAP_ERR_NUMERIC
                       : h[0] == kCheckPairCapacity ? TGAP_ERR_CAPACITY
                                                    : TGAP_ERR_CUDA;
    return set_error(ctx, status,
                     "device check %d (%s): index %d value %d, %d failure(s)", h[0], w, h[1], h[2], h[3]);
}

int sync_check_launch(tgap_context *ctx)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TGAP_CUDA(ctx, cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return TGAP_OK;
    return read_device_check(ctx);
}

}  // namespace tgap

extern "C" int tgap_synchronize(tgap_context *ctx)
{
    CHECK_RC(activate(ctx));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return read_device_check(ctx);
}

extern "C" const char *tgap_last_error(const tgap_context *ctx)
{
    return ctx ? ctx->last_error.c_str() : thread_error_text();
}

extern "C" int64_t tgap_kernel_launches(const tgap_context *ctx) { return ctx ? ctx->launches : 0; }

static void timing_collect(tgap_context *ctx)
{
    if (ctx->pending.empty()) return;
    cudaStreamSynchronize(ctx->stream);
    for (auto &r : ctx->pending) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, r.start, r.stop) == cudaSuccess) {
            ctx->stage_ms[r.stage] += ms;
            ctx->stage_count[r.stage] += 1;
        }
        ctx->event_pool.push_back(r.start);
        ctx->event_pool.push_back(r.stop);
    }
    ctx->pending.clear();
}

extern "C" int tgap_timing_enable(tgap_context *ctx, int enable)
{
    CHECK_RC(activate(ctx));
    if (!enable) timing_collect(ctx);
    ctx->timing = enable != 0;
    return TGAP_OK;
}

extern "C" int tgap_timing_reset(tgap_context *ctx)
{
    CHECK_RC(activate(ctx));
    timing_collect(ctx);
    for (auto &v : ctx->stage_ms) v = 0.0;
    for (auto &c : ctx->stage_count) c = 0;
    return TGAP_OK;
}

extern "C" int tgap_timing_report(tgap_context *ctx, int cap, char *names, double *total_ms, int64_t *counts,
                                  int *n_stages)
{
    CHECK_RC(activate(ctx));
    if (cap < 0 || !n_stages) return TGAP_ERR_ARGUMENT;
    timing_collect(ctx);
    const int n = (int)ctx->stage_names.size();
    *n_stages = n;
    for (int i = 0; i < n && i < cap; ++i) {
        if (names) {
            std::memset(names + 32 * i, 0, 32);
            std::strncpy(names + 32 * i, ctx->stage_names[i].c_str(), 31);
        }
        if (total_ms) total_ms[i] = ctx->stage_ms[i];
        if (counts) counts[i] = ctx->stage_count[i];
    }
    return TGAP_OK;
}

// ============================================================================ neighbors

extern "C" int tgap_number_of_unit_cells(const double a[3], const double b[3], const double c[3],
                                         double rcut, int indices[3])
{
    // neighbors_interface.f90:655-708 (host arithmetic, no contraction)
    if (!a || !b || !c || !indices) return TGAP_ERR_ARGUMENT;
    auto cross = [](const double *x, const double *y, double *z) {
        z[0] = x[1] * y[2] - x[2] * y[1];
        z[1] = x[2] * y[0] - x[0] * y[2];
        z[2] = x[0] * y[1] - x[1] * y[0];
    };
    auto dot = [](const double *x, const double *y) {
        double s = 0.0;
        s = s + x[0] * y[0];
        s = s + x[1] * y[1];
        s = s + x[2] * y[2];
        return s;
    };
    double axb[3], cxa[3], bxc[3];
    cross(a, b, axb);
    cross(c, a, cxa);
    cross(b, c, bxc);
    double n = std::sqrt(dot(axb, axb));
    for (double &v : axb) v = v / n;
    n = std::sqrt(dot(cxa, cxa));
    for (double &v : cxa) v = v / n;
    n = std::sqrt(dot(bxc, bxc));
    for (double &v : bxc) v = v / n;
    double m[3][3] = {{dot(axb, a), dot(axb, b), dot(axb, c)},
                      {dot(cxa, a), dot(cxa, b), dot(cxa, c)},
                      {dot(bxc, a), dot(bxc, b), dot(bxc, c)}};
    volatile double md = -m[0][2] * m[1][1] * m[2][0];
    md = md + m[0][1] * m[1][2] * m[2][0];
    md = md + m[0][2] * m[1][0] * m[2][1];
    md = md - m[0][0] * m[1][2] * m[2][1];
    md = md - m[0][1] * m[1][0] * m[2][2];
    md = md + m[0][0] * m[1][1] * m[2][2];
    double inv[3][3] = {{m[1][1] * m[2][2] - m[1][2] * m[2][1], m[0][2] * m[2][1] - m[0][1] * m[2][2],
                         m[0][1] * m[1][2] - m[0][2] * m[1][1]},
                        {m[1][2] * m[2][0] - m[1][0] * m[2][2], m[0][0] * m[2][2] - m[0][2] * m[2][0],
                         m[0][2] * m[1][0] - m[0][0] * m[1][2]},
                        {m[1][0] * m[2][1] - m[1][1] * m[2][0], m[0][1] * m[2][0] - m[0][0] * m[2][1],
                         m[0][0] * m[1][1] - m[0][1] * m[1][0]}};
    const double v = 2.0 * rcut;
    for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s = s + (inv[i][k] / md) * v;
        double ir = std::fabs(s);
        indices[i] = (int)ir;
        if (ir > (double)indices[i]) indices[i] += 1;
    }
    return TGAP_OK;
}

extern "C" int tgap_build_neighbors(tgap_context *ctx, int n_sites, int n_sites_supercell,
                                    const double *positions, const double a_box[3],
                                    const double b_box[3], const double c_box[3], int box_small,
                                    double rcut_max, const int *species_supercell, int rebuild,
                                    int *n_neigh, int *neighbors_list, double *rjs, double *xyz,
                                    double *thetas, double *phis, int *neighbor_species,
                                    int64_t capacity, int64_t *n_atom_pairs)
{
    CHECK_RC(activate(ctx));
    if (n_sites < 0 || n_sites_supercell < n_sites || !positions || !a_box || !b_box || !c_box ||
        !n_neigh || !neighbors_list || !n_atom_pairs || !(rcut_max > 0))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_build_neighbors: bad arguments");
    NeighborBatch nb;
    std::unique_ptr<NeighborBatch, void (*)(NeighborBatch *)> guard(&nb, [](NeighborBatch *p) { p->release_all(); });
    CHECK_RC(neighbors_setup_supercell(ctx, &nb, n_sites, n_sites_supercell, positions, a_box, b_box,
                                       c_box, box_small, rcut_max, species_supercell));
    int64_t P = 0;
    if (rebuild) {
        int rc = neighbors_build(ctx, &nb, 1, capacity, &P, true);
        *n_atom_pairs = P;
        if (rc == TGAP_ERR_CAPACITY)
            return set_error(ctx, rc, "neighbor capacity %lld < %lld pairs", (long long)capacity,
                             (long long)P);
        if (rc) return rc;
    } else {
        // geometry refresh of the caller's list
        P = 0;
        for (int i = 0; i < n_sites; ++i) P += n_neigh[i];
        if (P > capacity) return set_error(ctx, TGAP_ERR_CAPACITY, "capacity");
        if (nb.ensure_pairs(P)) return set_error(ctx, TGAP_ERR_NOMEM, "pairs");
        nb.n_pairs = P;
        CHECK_RC(upload(ctx, nb.n_neigh, n_neigh, (size_t)n_sites));
        CHECK_RC(upload(ctx, nb.list, neighbors_list, (size_t)P));
        CHECK_RC(neighbors_set_counts(ctx, &nb));
        int64_t dummy = 0;
        CHECK_RC(neighbors_build(ctx, &nb, 0, capacity, &dummy, true));
        *n_atom_pairs = P;
    }
    CHECK_RC(download(ctx, n_neigh, nb.n_neigh, (size_t)n_sites));
    CHECK_RC(download(ctx, neighbors_list, nb.list, (size_t)P));
    if (rjs) CHECK_RC(download(ctx, rjs, nb.rjs, (size_t)P));
    if (xyz) CHECK_RC(download(ctx, xyz, nb.xyz, 3 * (size_t)P));
    if (thetas) CHECK_RC(download(ctx, thetas, nb.thetas, (size_t)P));
    if (phis) CHECK_RC(download(ctx, phis, nb.phis, (size_t)P));
    if (neighbor_species) CHECK_RC(download(ctx, neighbor_species, nb.nspecies, (size_t)P));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

// ============================================================================ descriptor

static int hypers_from_args(int n_species, const int *alpha_max, int l_max, const double *rcut_hard,
                            const double *rcut_soft, const double *nf, const double *global_scaling,
                            const double *atom_sigma_r, const double *atom_sigma_r_scaling,
                            const double *atom_sigma_t, const double *atom_sigma_t_scaling,
                            const double *amplitude_scaling, int radial_enhancement,
                            const double *central_weight, tgap_soap_hypers *h)
{
    if (!alpha_max || !rcut_hard || !rcut_soft || !nf || !global_scaling || !atom_sigma_r ||
        !atom_sigma_r_scaling || !atom_sigma_t || !atom_sigma_t_scaling || !amplitude_scaling ||
        !central_weight)
        return TGAP_ERR_ARGUMENT;
    h->n_species = n_species;
    h->alpha_max = alpha_max;
    h->l_max = l_max;
    h->rcut_hard = rcut_hard;
    h->rcut_soft = rcut_soft;
    h->nf = nf;
    h->global_scaling = global_scaling;
    h->atom_sigma_r = atom_sigma_r;
    h->atom_sigma_r_scaling = atom_sigma_r_scaling;
    h->atom_sigma_t = atom_sigma_t;
    h->atom_sigma_t_scaling = atom_sigma_t_scaling;
    h->amplitude_scaling = amplitude_scaling;
    h->central_weight = central_weight;
    h->radial_enhancement = radial_enhancement;
    return TGAP_OK;
}

static int prepare_soap(tgap_context *ctx, const tgap_soap_hypers *h, DeviceSoap *ds)
{
    SoapParams p;
    std::string why;
    int rc = make_soap_params(h, &p, &why);
    if (rc) return set_error(ctx, rc, "descriptor hypers: %s", why.c_str());
    SoapTables t;
    build_soap_tables(p, &t);
    return upload_soap(ctx, p, t, ds);
}

static void release_soap(DeviceSoap *ds)
{
    ds->xq.release();
    ds->tq.release();
    ds->central.release();
    ds->xq32.release();
    ds->tq32.release();
    ds->central32.release();
    ds->rtab.release();
    ds->cmp_i.release();
    ds->cmp_f64.release();
    ds->cmp_f32.release();
}

// The compression P (entries P_i, P_j 1-based, values P_el) of a model's descriptor on the device:
// CSR by output component and CSC by power-spectrum component, each in the given entry order.
static int upload_compression(tgap_context *ctx, DeviceSoap *ds, int dim_out, int nnz, const int *P_i,
                              const int *P_j, const double *P_el)
{
    const int dim = ds->p.dim;
    if (dim_out <= 0 || nnz <= 0 || !P_i || !P_j || !P_el)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "compression: bad arguments");
    for (int e = 0; e < nnz; ++e)
        if (P_i[e] < 1 || P_i[e] > dim_out || P_j[e] < 1 || P_j[e] > dim)
            return set_error(ctx, TGAP_ERR_ARGUMENT, "compression entry %d (%d, %d) outside %d x %d", e, P_i[e],
                             P_j[e], dim_out, dim);
    std::vector<int> row(dim_out + 1, 0), col(dim + 1, 0), rcol(nnz), crow(nnz);
    std::vector<double> rval(nnz), cval(nnz);
    for (int e = 0; e < nnz; ++e) {
        ++row[P_i[e]];
        ++col[P_j[e]];
    }
    for (int r = 0; r < dim_out; ++r) row[r + 1] += row[r];
    for (int c = 0; c < dim; ++c) col[c + 1] += col[c];
    std::vector<int> rfill(row.begin(), row.end() - 1), cfill(col.begin(), col.end() - 1);
    for (int e = 0; e < nnz; ++e) {
        const int r = P_i[e] - 1, c = P_j[e] - 1;
        rcol[rfill[r]] = c;
        rval[rfill[r]++] = P_el[e];
        crow[cfill[c]] = r;
        cval[cfill[c]++] = P_el[e];
    }
    // one int buffer [row | rcol | col | crow], one FP64 and one FP32 buffer [rval | cval]
    std::vector<int> ib;
    ib.insert(ib.end(), row.begin(), row.end());
    ib.insert(ib.end(), rcol.begin(), rcol.end());
    ib.insert(ib.end(), col.begin(), col.end());
    ib.insert(ib.end(), crow.begin(), crow.end());
    std::vector<double> db(rval);
    db.insert(db.end(), cval.begin(), cval.end());
    std::vector<float> fb(db.begin(), db.end());
    CHECK_RC(upload(ctx, ds->cmp_i, ib.data(), ib.size()));
    CHECK_RC(upload(ctx, ds->cmp_f64, db.data(), db.size()));
    CHECK_RC(upload(ctx, ds->cmp_f32, fb.data(), fb.size()));
    const int *i0 = ds->cmp_i.as<int>();
    ds->p.dim_out = dim_out;
    ds->p.cmp_row = i0;
    ds->p.cmp_rcol = i0 + dim_out + 1;
    ds->p.cmp_col = i0 + dim_out + 1 + nnz;
    ds->p.cmp_crow = i0 + dim_out + 1 + nnz + dim + 1;
    ds->p.cmp_rval = ds->cmp_f64.as<double>();
    ds->p.cmp_cval = ds->cmp_f64.as<double>() + nnz;
    ds->p.cmp_rval32 = ds->cmp_f32.as<float>();
    ds->p.cmp_cval32 = ds->cmp_f32.as<float>() + nnz;
    return TGAP_OK;
}

extern "C" int tgap_get_soap(tgap_context *ctx, int n_sites, const int *n_neigh, int n_species,
                             const int *species, const int *species_multiplicity, int n_atom_pairs,
                             const unsigned char *mask, const double *rjs, const double *thetas,
                             const double *phis, const int *alpha_max, int l_max,
                             const double *rcut_hard, const double *rcut_soft, const double *nf,
                             const double *global_scaling, const double *atom_sigma_r,
                             const double *atom_sigma_r_scaling, const double *atom_sigma_t,
                             const double *atom_sigma_t_scaling, const double *amplitude_scaling,
                             int radial_enhancement, const double *central_weight, const char *basis,
                             const char *scaling_mode, int do_derivatives, int compress_soap,
                             int compress_P_nonzero, const int *compress_P_i, const int *compress_P_j,
                             const double *compress_P_el, double *soap, double *soap_cart_der)
{
    CHECK_RC(activate(ctx));
    (void)species;
    if (n_sites < 0 || n_atom_pairs < n_sites || !n_neigh || !mask || !rjs || !thetas || !phis || !soap)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_soap: bad arguments");
    if (basis && std::strncmp(basis, "poly3", 5) == 0 && std::strncmp(basis, "poly3gauss", 10) == 0)
        return set_error(ctx, TGAP_ERR_UNSUPPORTED, "basis poly3gauss is not implemented");
    if (basis && std::strncmp(basis, "poly3", 5) != 0)
        return set_error(ctx, TGAP_ERR_UNSUPPORTED, "basis must be poly3");
    if (scaling_mode && std::strncmp(scaling_mode, "polynomial", 10) != 0)
        return set_error(ctx, TGAP_ERR_UNSUPPORTED, "scaling_mode must be polynomial");
    if (species_multiplicity)
        for (int i = 0; i < n_sites; ++i)
            if (species_multiplicity[i] > 1)
                return set_error(ctx, TGAP_ERR_UNSUPPORTED, "species multiplicity > 1");
    tgap_soap_hypers h;
    if (hypers_from_args(n_species, alpha_max, l_max, rcut_hard, rcut_soft, nf, global_scaling,
                         atom_sigma_r, atom_sigma_r_scaling, atom_sigma_t, atom_sigma_t_scaling,
                         amplitude_scaling, radial_enhancement, central_weight, &h))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_soap: null hyperparameter array");
    DeviceSoap ds;
    std::unique_ptr<DeviceSoap, void (*)(DeviceSoap *)> g0(&ds, release_soap);
    CHECK_RC(prepare_soap(ctx, &h, &ds));
    const SoapParams &P = ds.p;
    // pair arrays: xyz from (r, theta, phi), species channel from the mask
    const size_t np = (size_t)n_atom_pairs;
    std::vector<double> hxyz(3 * np);
    std::vector<int> hsp(np, 0);
    std::vector<int64_t> hstart(n_sites + 1, 0);
    for (int i = 0; i < n_sites; ++i) hstart[i + 1] = hstart[i] + n_neigh[i];
    if (hstart[n_sites] != n_atom_pairs)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "sum(n_neigh) != n_atom_pairs");
    for (size_t k = 0; k < np; ++k) {
        const double r = rjs[k], st = std::sin(thetas[k]);
        hxyz[3 * k] = r * st * std::cos(phis[k]);
        hxyz[3 * k + 1] = r * st * std::sin(phis[k]);
        hxyz[3 * k + 2] = r * std::cos(thetas[k]);
        for (int s = 0; s < n_species; ++s)
            if (mask[k + np * s]) {
                hsp[k] = s + 1;
                break;
            }
    }
    DevBuf *S = ctx->scratch;
    CHECK_RC(upload(ctx, S[0], hstart.data(), hstart.size()));
    CHECK_RC(upload(ctx, S[1], hxyz.data(), hxyz.size()));
    CHECK_RC(upload(ctx, S[2], rjs, np));
    CHECK_RC(upload(ctx, S[3], hsp.data(), np));
    const int nlm = (P.l_max + 1) * (P.l_max + 1);
    if (S[4].ensure(sizeof(double) * (size_t)n_sites * P.n_max * nlm + 8) ||
        S[5].ensure(sizeof(double) * (size_t)n_sites * P.dim + 8) ||
        S[6].ensure(sizeof(double) * (size_t)n_sites + 8))
        return set_error(ctx, TGAP_ERR_NOMEM, "descriptor workspace");
    PairView pv{S[0].as<int64_t>(), S[1].as<double>(), S[2].as<double>(), S[3].as<int>(), nullptr, 0,
                ctx->d_check};
    SoapOut o;
    o.c = S[4].ptr;
    o.q = S[5].ptr;
    o.norm = S[6].ptr;
    o.q_ld = P.dim;
    const bool der = do_derivatives && soap_cart_der;
    CHECK_RC(soap_forward(ctx, ds, pv, nullptr, n_sites, TGAP_FP64, o));
    if (der) {
        if (S[7].ensure(sizeof(double) * 3 * (size_t)P.dim * np + 8))
            return set_error(ctx, TGAP_ERR_NOMEM, "soap_cart_der (%zu bytes)",
                             sizeof(double) * 3 * (size_t)P.dim * np);
        CHECK_RC(tgap::soap_cart_der(ctx, ds, pv, nullptr, n_sites, o, S[7].as<double>()));
    }
    if (!compress_soap) {
        CHECK_RC(download(ctx, soap, S[5], (size_t)n_sites * P.dim));
        if (der) CHECK_RC(download(ctx, soap_cart_der, S[7], 3 * (size_t)P.dim * np));
    } else {
        // the compression (soap is then n_soap = dim_out x n_sites): the uncompressed q and
        // derivatives above mapped by P (the launches above already hold the uncompressed params)
        int dim_out = 0;
        for (int e = 0; e < compress_P_nonzero; ++e) dim_out = std::max(dim_out, compress_P_i ? compress_P_i[e] : 0);
        CHECK_RC(upload_compression(ctx, &ds, dim_out, compress_P_nonzero, compress_P_i, compress_P_j, compress_P_el));
        if (S[8].ensure(sizeof(double) * (size_t)n_sites * dim_out + 8) ||
            (der && S[9].ensure(sizeof(double) * 3 * (size_t)dim_out * np + 8)))
            return set_error(ctx, TGAP_ERR_NOMEM, "compressed descriptor");
        CHECK_RC(soap_compress_rows(ctx, ds, n_sites, S[0].as<int64_t>(), S[5].as<double>(),
                                    der ? S[7].as<double>() : nullptr, S[8].as<double>(),
                                    der ? S[9].as<double>() : nullptr));
        CHECK_RC(download(ctx, soap, S[8], (size_t)n_sites * dim_out));
        if (der) CHECK_RC(download(ctx, soap_cart_der, S[9], 3 * (size_t)dim_out * np));
    }
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

extern "C" int tgap_get_soap_energy_and_forces(tgap_context *ctx, int n_soap, int n_sites,
                                               int n_sparse, const double *soap,
                                               const double *soap_der, const double *alphas,
                                               double delta, double zeta0, double e0,
                                               const double *Qs, const int *n_neigh,
                                               const int *neighbors_list, const double *xyz,
                                               int n_atom_pairs, int do_forces, int n_sites0,
                                               double *energies, double *forces, double *virial)
{
    CHECK_RC(activate(ctx));
    if (n_soap <= 0 || n_sites < 0 || n_sparse <= 0 || !soap || !alphas || !Qs || !energies ||
        (do_forces && (!soap_der || !n_neigh || !neighbors_list || !xyz || !forces || !virial ||
                       n_sites0 <= 0)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_soap_energy_and_forces: bad arguments");
    DeviceModel m;
    m.n_sparse = n_sparse;
    m.dim = n_soap;
    m.delta = delta;
    m.zeta = zeta0;
    DevBuf *S = ctx->scratch;
    CHECK_RC(upload(ctx, m.Qs, Qs, (size_t)n_sparse * n_soap));
    CHECK_RC(upload(ctx, m.alphas, alphas, (size_t)n_sparse));
    if (m.QsT.ensure(sizeof(double) * (size_t)n_sparse * n_soap))
        return set_error(ctx, TGAP_ERR_NOMEM, "Qs transpose");
    CHECK_RC(transpose_f64(ctx, n_sparse, n_soap, m.Qs.as<double>(), m.QsT.as<double>()));
    CHECK_RC(upload(ctx, S[0], soap, (size_t)n_sites * n_soap));
    if (S[1].ensure(sizeof(double) * (size_t)(n_sites + 1))) return TGAP_ERR_NOMEM;
    GapWork w;
    int rc = gap_energy_grad_f64(ctx, m, S[0].as<double>(), n_soap, n_sites, e0, do_forces, &w, nullptr,
                                 S[1].as<double>(), nullptr);
    if (!rc) rc = download(ctx, energies, S[1], (size_t)n_sites);
    if (!rc && do_forces) {
        std::vector<int64_t> hstart(n_sites + 1, 0);
        for (int i = 0; i < n_sites; ++i) hstart[i + 1] = hstart[i] + n_neigh[i];
        const size_t P = (size_t)hstart[n_sites];
        if ((int64_t)P != (int64_t)n_atom_pairs) rc = set_error(ctx, TGAP_ERR_ARGUMENT, "sum(n_neigh) != n_atom_pairs");
        if (!rc) rc = upload(ctx, S[2], hstart.data(), hstart.size());
        if (!rc) rc = upload(ctx, S[3], neighbors_list, P);
        if (!rc) rc = upload(ctx, S[4], soap_der, 3 * P * (size_t)n_soap);
        if (!rc) rc = upload(ctx, S[5], xyz, 3 * P);
        if (!rc && (S[6].ensure(sizeof(double) * 3 * (size_t)n_sites0) || S[7].ensure(sizeof(double) * 9)))
            rc = TGAP_ERR_NOMEM;
        if (!rc) {
            cudaMemsetAsync(S[6].ptr, 0, sizeof(double) * 3 * (size_t)n_sites0, ctx->stream);
            cudaMemsetAsync(S[7].ptr, 0, sizeof(double) * 9, ctx->stream);
            rc = pair_forces_from_der(ctx, n_sites, S[2].as<int64_t>(), S[3].as<int>(), n_sites0,
                                      w.g.as<double>(), n_soap, S[4].as<double>(), S[5].as<double>(),
                                      S[6].as<double>(), S[7].as<double>());
        }
        if (!rc) rc = download(ctx, forces, S[6], 3 * (size_t)n_sites0);
        if (!rc) rc = download(ctx, virial, S[7], 9);
    }
    if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? TGAP_OK : TGAP_ERR_CUDA;
    m.Qs.release();
    m.QsT.release();
    m.alphas.release();
    w.e_part.release();
    w.G.release();
    w.g.release();
    return rc;
}

extern "C" int tgap_local_property_predict(tgap_context *ctx, int n_soap, int n_sites, int n_sparse,
                                           const double *soap, const double *Qs, const double *alphas, double V0,
                                           double delta, double zeta, int do_derivatives,
                                           const double *soap_cart_der, const int *n_neigh, int n_atom_pairs,
                                           double *V, double *V_der)
{
    CHECK_RC(activate(ctx));
    if (n_soap <= 0 || n_sites < 0 || n_sparse <= 0 || !soap || !Qs || !alphas || !V ||
        (do_derivatives && (!soap_cart_der || !n_neigh || !V_der || n_atom_pairs < 0)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_local_property_predict: bad arguments");
    if (n_sites == 0) return TGAP_OK;
    DeviceModel m;
    m.n_sparse = n_sparse;
    m.dim = n_soap;
    m.delta = delta;
    m.zeta = zeta;
    m.zeta_tol = 1.0e-10;  // local_properties.f90:76-77
    m.zeta_nint = true;
    DevBuf *S = ctx->scratch;
    GapWork w;
    auto cleanup = [&]() {
        m.Qs.release();
        m.QsT.release();
        m.alphas.release();
        w.e_part.release();
        w.G.release();
        w.g.release();
    };
    int rc = upload(ctx, m.Qs, Qs, (size_t)n_sparse * n_soap);
    if (!rc) rc = upload(ctx, m.alphas, alphas, (size_t)n_sparse);
    if (!rc && m.QsT.ensure(sizeof(double) * (size_t)n_sparse * n_soap)) rc = set_error(ctx, TGAP_ERR_NOMEM, "Qs transpose");
    if (!rc) rc = transpose_f64(ctx, n_sparse, n_soap, m.Qs.as<double>(), m.QsT.as<double>());
    if (!rc) rc = upload(ctx, S[0], soap, (size_t)n_sites * n_soap);
    if (!rc && S[1].ensure(sizeof(double) * (size_t)n_sites)) rc = TGAP_ERR_NOMEM;
    // V = delta^2 K^zeta alphas + V0 (the GAP energy with e0 = V0), clipped; g = dV/dq
    if (!rc)
        rc = gap_energy_grad_f64(ctx, m, S[0].as<double>(), n_soap, n_sites, V0, do_derivatives, &w, nullptr,
                                 S[1].as<double>(), nullptr);
    if (!rc) rc = clip_nonneg(ctx, n_sites, S[1].as<double>());
    if (!rc) rc = download(ctx, V, S[1], (size_t)n_sites);
    if (!rc && do_derivatives) {
        std::vector<int64_t> hstart(n_sites + 1, 0);
        for (int i = 0; i < n_sites; ++i) hstart[i + 1] = hstart[i] + n_neigh[i];
        const size_t P = (size_t)hstart[n_sites];
        if ((int64_t)P != (int64_t)n_atom_pairs) rc = set_error(ctx, TGAP_ERR_ARGUMENT, "sum(n_neigh) != n_atom_pairs");
        if (!rc && P > 0) {
            rc = upload(ctx, S[2], hstart.data(), hstart.size());
            if (!rc) rc = upload(ctx, S[4], soap_cart_der, 3 * P * (size_t)n_soap);
            if (!rc && S[6].ensure(sizeof(double) * 3 * P)) rc = TGAP_ERR_NOMEM;
            if (!rc)
                rc = local_property_pairs(ctx, n_sites, S[2].as<int64_t>(), w.g.as<double>(), n_soap, S[4].as<double>(),
                                          S[1].as<double>(), S[6].as<double>());
            if (!rc) rc = download(ctx, V_der, S[6], 3 * P);
        }
    }
    if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? TGAP_OK : TGAP_ERR_CUDA;
    cleanup();
    return rc ? rc : read_device_check(ctx);
}

extern "C" int tgap_assign_species(int n_species, const char *species_types, int n, const char *names,
                                   int *out)
{
    if (n_species <= 0 || !species_types || n < 0 || (n > 0 && (!names || !out))) return TGAP_ERR_ARGUMENT;
    auto trimmed = [](const char *p) {
        std::string s(p, 8);
        while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
        return s;
    };
    for (int a = 0; a < n_species; ++a)
        for (int b = a + 1; b < n_species; ++b)
            if (trimmed(species_types + 8 * a) == trimmed(species_types + 8 * b)) return TGAP_ERR_UNSUPPORTED;
    for (int i = 0; i < n; ++i) {
        out[i] = 0;
        std::string nm = trimmed(names + 8 * (size_t)i);
        for (int s = 0; s < n_species; ++s)
            if (trimmed(species_types + 8 * s) == nm) {
                out[i] = s + 1;
                break;
            }
    }
    return TGAP_OK;
}

// ============================================================================ resident objects

struct tgap_model {
    tgap_context *ctx;
    DeviceSoap soap;
    DeviceModel gap;
    int central_species;
    bool mixed_ready = false;
};

struct SiteSet {
    int central_species = -1;
    int n_rows = 0;
    DevBuf sites;
};

struct tgap_system {
    tgap_context *ctx;
    NeighborBatch nb;
    double rcut;
    std::vector<int> host_species;
    DevBuf d_species;  // species channel per site (pair and triplet terms), uploaded on first use
    DevBuf queue;      // site counters of the persistent descriptor launches (kQueueInts)
    std::vector<SiteSet> site_sets;
    DevBuf c, q, norm, q_hi, q_lo, e_rows;
    GapWork gw;
    DevBuf scratch_forces;
    // per-atom isolated-atom energies (calculate_e0), added to every energy output when set
    std::vector<double> host_e0;
    DevBuf d_e0;
    // sites evaluated as descriptor centres: atoms [range_beg, range_end) (split_tasks of one rank)
    int range_beg = 0, range_end = -1;
    // device work of the host-buffer entry as CUDA graphs, one per call configuration
    struct CallGraph {
        std::vector<const tgap_model *> models;
        int precision = 0, flags = 0;
        const void *io[4] = {nullptr, nullptr, nullptr, nullptr};
        bool seen = false;  // ran eagerly once at seen_epoch (buffers sized): the next call captures
        uint64_t seen_epoch = 0;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        uint64_t epoch = 0;
        int64_t kernels = 0;
    };
    std::vector<CallGraph> call_graphs;
};

static int model_create(tgap_context *ctx, const tgap_soap_hypers *hypers, int central_species, int n_sparse,
                        const double *alphas, const double *Qs, double delta, double zeta, int dim_out,
                        int P_nonzero, const int *P_i, const int *P_j, const double *P_el, tgap_model **out)
{
    CHECK_RC(activate(ctx));
    if (!hypers || n_sparse <= 0 || !alphas || !Qs || !out)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_model_create: bad arguments");
    auto *m = new tgap_model();
    m->ctx = ctx;
    m->central_species = central_species;
    int rc = prepare_soap(ctx, hypers, &m->soap);
    if (!rc && P_nonzero > 0) rc = upload_compression(ctx, &m->soap, dim_out, P_nonzero, P_i, P_j, P_el);
    if (!rc) {
        m->gap.n_sparse = n_sparse;
        m->gap.dim = m->soap.p.dim_out;  // the descriptor's length, compressed or not
        m->gap.delta = delta;
        m->gap.zeta = zeta;
        rc = upload(ctx, m->gap.Qs, Qs, (size_t)n_sparse * m->gap.dim);
    }
    if (!rc) rc = upload(ctx, m->gap.alphas, alphas, (size_t)n_sparse);
    if (!rc && m->gap.QsT.ensure(sizeof(double) * (size_t)n_sparse * m->gap.dim)) rc = TGAP_ERR_NOMEM;
    if (!rc) rc = transpose_f64(ctx, n_sparse, m->gap.dim, m->gap.Qs.as<double>(), m->gap.QsT.as<double>());
    if (!rc) rc = model_upload_mixed(ctx, &m->gap);
    if (!rc) m->mixed_ready = true;
    if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = TGAP_ERR_CUDA;
    if (rc) {
        tgap_model_destroy(m);
        return rc;
    }
    *out = m;
    return TGAP_OK;
}

extern "C" int tgap_model_create(tgap_context *ctx, const tgap_soap_hypers *hypers, int central_species,
                                 int n_sparse, const double *alphas, const double *Qs, double delta,
                                 double zeta, tgap_model **out)
{
    return model_create(ctx, hypers, central_species, n_sparse, alphas, Qs, delta, zeta, 0, 0, nullptr, nullptr,
                        nullptr, out);
}

extern "C" int tgap_model_create_compressed(tgap_context *ctx, const tgap_soap_hypers *hypers, int central_species,
                                            int n_sparse, const double *alphas, const double *Qs, double delta,
                                            double zeta, int dim_out, int P_nonzero, const int *P_i,
                                            const int *P_j, const double *P_el, tgap_model **out)
{
    if (P_nonzero <= 0) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_model_create_compressed: no entries");
    return model_create(ctx, hypers, central_species, n_sparse, alphas, Qs, delta, zeta, dim_out, P_nonzero, P_i,
                        P_j, P_el, out);
}

extern "C" int tgap_model_destroy(tgap_model *m)
{
    if (!m) return TGAP_OK;
    cudaSetDevice(m->ctx->device);
    release_soap(&m->soap);
    DevBuf *bufs[] = {&m->gap.Qs, &m->gap.QsT, &m->gap.alphas, &m->gap.alphas32, &m->gap.Q_hi,
                      &m->gap.Q_lo, &m->gap.QT_hi, &m->gap.QT_lo};
    for (DevBuf *b : bufs) b->release();
    delete m;
    return TGAP_OK;
}

extern "C" int tgap_model_dim(const tgap_model *m) { return m ? m->gap.dim : 0; }

extern "C" int tgap_system_create(tgap_context *ctx, int n_structures, const int *offsets,
                                  const double *positions, const double *boxes, const int *species,
                                  double rcut_max, tgap_system **out)
{
    CHECK_RC(activate(ctx));
    if (n_structures <= 0 || !offsets || !positions || !boxes || !species || !out || !(rcut_max > 0))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_system_create: bad arguments");
    auto *s = new tgap_system();
    s->ctx = ctx;
    s->rcut = rcut_max;
    s->host_species.assign(species, species + offsets[n_structures]);
    int rc = neighbors_setup(ctx, &s->nb, n_structures, offsets, positions, boxes, species, rcut_max,
                             nullptr);
    if (!rc) rc = tgap_system_update(s, 1);
    if (rc) {
        tgap_system_destroy(s);
        return rc;
    }
    *out = s;
    return TGAP_OK;
}

extern "C" int tgap_system_destroy(tgap_system *s)
{
    if (!s) return TGAP_OK;
    cudaSetDevice(s->ctx->device);
    s->nb.release_all();
    for (auto &ss : s->site_sets) ss.sites.release();
    for (auto &cg : s->call_graphs) {
        if (cg.exec) cudaGraphExecDestroy(cg.exec);
        if (cg.graph) cudaGraphDestroy(cg.graph);
    }
    DevBuf *bufs[] = {&s->c, &s->q, &s->norm, &s->q_hi, &s->q_lo, &s->e_rows, &s->gw.e_part, &s->gw.G,
                      &s->gw.g, &s->gw.G_hi, &s->gw.G_lo, &s->scratch_forces, &s->d_species, &s->queue,
                      &s->d_e0};
    for (DevBuf *b : bufs) b->release();
    delete s;
    return TGAP_OK;
}

extern "C" int tgap_system_n_atoms(const tgap_system *s) { return s ? s->nb.n_atoms : 0; }
extern "C" int64_t tgap_system_n_pairs(const tgap_system *s)
{
    if (!s) return 0;
    // after device-side rebuilds (MD) the count is read back here
    tgap_system *m = const_cast<tgap_system *>(s);
    if (m->nb.count_on_device && (activate(m->ctx) || neighbors_sync_count(m->ctx, &m->nb))) return -1;
    return s->nb.n_pairs;
}

extern "C" int tgap_system_positions(tgap_system *s, double **d_positions)
{
    if (!s || !d_positions) return TGAP_ERR_ARGUMENT;
    *d_positions = s->nb.positions.as<double>();
    return TGAP_OK;
}

extern "C" int tgap_system_get_positions(tgap_system *s, double *positions)
{
    if (!s || !positions) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = s->ctx;
    CHECK_RC(activate(ctx));
    TGAP_CUDA(ctx, cudaMemcpyAsync(positions, s->nb.positions.ptr, sizeof(double) * 3 * s->nb.n_atoms,
                                   cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

extern "C" int tgap_system_set_positions(tgap_system *s, const double *positions)
{
    if (!s || !positions) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = s->ctx;
    CHECK_RC(activate(ctx));
    TGAP_CUDA(ctx, cudaMemcpyAsync(s->nb.positions.ptr, positions, sizeof(double) * 3 * s->nb.n_atoms,
                                   cudaMemcpyHostToDevice, ctx->stream));
    return TGAP_OK;
}

// split_tasks (misc.f90:88-111) on the device side: only atoms [beg, end) are descriptor centres of
// later evaluations; their energies, and their force and virial contributions on every atom they
// see, are computed (the other energies are 0), as one rank of the reference's MPI split does before
// collect_calculation (mpi_utils.f90:515-545) sums the ranks.
extern "C" int tgap_system_set_site_range(tgap_system *s, int beg, int end)
{
    graphs_stale();
    if (!s) return TGAP_ERR_ARGUMENT;
    const int N = (int)s->host_species.size();
    if (end < 0) end = N;
    if (beg < 0 || beg > end || end > N) return set_error(s->ctx, TGAP_ERR_ARGUMENT, "site range [%d, %d) of %d", beg, end, N);
    CHECK_RC(activate(s->ctx));
    TGAP_CUDA(s->ctx, cudaStreamSynchronize(s->ctx->stream));
    for (auto &ss : s->site_sets) ss.sites.release();  // rebuilt for the new range on next use
    s->site_sets.clear();
    s->range_beg = beg;
    s->range_end = end == N ? -1 : end;
    return TGAP_OK;
}

// velocity_verlet (md_utils.f90:486-532) on device arrays, for drivers that assemble the forces
// themselves (for example summed over ranks): masses in eV fs^2 / A^2.
extern "C" int tgap_velocity_verlet(tgap_context *ctx, int n_sites, double *d_positions, double *d_positions_prev,
                                    double *d_velocities, const double *d_forces, double *d_forces_prev,
                                    const double *d_masses, double dt, double dt_prev, int first_step)
{
    CHECK_RC(activate(ctx));
    if (n_sites < 0 || (n_sites > 0 && (!d_positions || !d_positions_prev || !d_velocities || !d_forces ||
                                        !d_forces_prev || !d_masses)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_velocity_verlet: bad arguments");
    return velocity_verlet(ctx, n_sites, d_positions, d_positions_prev, d_velocities, d_forces, d_forces_prev,
                           d_masses, dt, dt_prev, first_step);
}

extern "C" int tgap_velocity_verlet_host(int n_sites, double *positions, double *positions_prev, double *velocities,
                                         const double *forces, double *forces_prev, const double *masses, double dt,
                                         double dt_prev, int first_step)
{
    if (n_sites < 0 || (n_sites > 0 && (!positions || !velocities || !forces || !forces_prev || !masses)))
        return TGAP_ERR_ARGUMENT;
    const size_t n3 = 3 * (size_t)n_sites;
    // non-finite forces: an exponent field of all ones, as one branch-free pass
    uint64_t bad = 0;
    for (size_t g = 0; g < n3; ++g) {
        uint64_t b;
        std::memcpy(&b, forces + g, sizeof(b));
        bad |= (uint64_t)(((b >> 52) & 0x7ff) == 0x7ff);
    }
    if (bad) return TGAP_ERR_NUMERIC;
    // one reciprocal mass per atom instead of a division per component (within an ulp of the
    // divided form); atoms in pairs, whose six components are three 2-wide vectors
    typedef double v2d __attribute__((vector_size(16)));
    const auto ld = [](const double *p) {
        v2d v;
        std::memcpy(&v, p, sizeof(v));
        return v;
    };
    const auto st = [](double *p, v2d v) { std::memcpy(p, &v, sizeof(v)); };
    const double hv = first_step ? 0.0 : 0.5 * dt_prev, hx = 0.5 * (dt * dt);
    const v2d vdt = {dt, dt};
    int i = 0;
    for (; i + 1 < n_sites; i += 2) {
        const double im0 = 1.0 / masses[i], im1 = 1.0 / masses[i + 1];
        const double cv0 = hv * im0, cv1 = hv * im1, cx0 = hx * im0, cx1 = hx * im1;
        const v2d cv[3] = {{cv0, cv0}, {cv0, cv1}, {cv1, cv1}}, cx[3] = {{cx0, cx0}, {cx0, cx1}, {cx1, cx1}};
        for (int k = 0; k < 3; ++k) {
            const size_t g = 3 * (size_t)i + 2 * k;
            const v2d fg = ld(forces + g);
            const v2d v = ld(velocities + g) + (fg + ld(forces_prev + g)) * cv[k];
            st(velocities + g, v);
            const v2d x = ld(positions + g);
            if (positions_prev) st(positions_prev + g, x);
            st(forces_prev + g, fg);
            st(positions + g, x + v * vdt + fg * cx[k]);
        }
    }
    for (; i < n_sites; ++i) {
        const double im = 1.0 / masses[i];
        const double cv = hv * im, cx = hx * im;
        for (int c = 0; c < 3; ++c) {
            const size_t g = 3 * (size_t)i + c;
            const double fg = forces[g];
            const double v = velocities[g] + (fg + forces_prev[g]) * cv;
            velocities[g] = v;
            const double x = positions[g];
            if (positions_prev) positions_prev[g] = x;
            forces_prev[g] = fg;
            positions[g] = x + v * dt + fg * cx;
        }
    }
    return TGAP_OK;
}

// calculate_e0 (calculate_gap_soap.f90:135-169): every atom gets the e0 of its species (the input
// file's e0 keyword, read_files.f90:380-385); atoms of no listed species keep 0.
extern "C" int tgap_system_set_e0(tgap_system *s, int n_species, const double *e0)
{
    graphs_stale();
    if (!s || n_species < 0 || (n_species > 0 && !e0)) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = s->ctx;
    CHECK_RC(activate(ctx));
    const size_t N = s->host_species.size();
    std::vector<double> v(N, 0.0);
    for (size_t i = 0; i < N; ++i) {
        const int sp = s->host_species[i];
        if (sp >= 1 && sp <= n_species) v[i] = e0[sp - 1];
    }
    CHECK_RC(upload(ctx, s->d_e0, v.data(), N));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    s->host_e0.swap(v);
    return TGAP_OK;
}

__global__ void k_add_e0(int beg, int end, const double *__restrict__ e0, double *__restrict__ energies)
{
    const int i = beg + blockIdx.x * blockDim.x + threadIdx.x;
    if (i < end) energies[i] += e0[i];
}

extern "C" int tgap_system_update(tgap_system *s, int rebuild)
{
    if (!s) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = s->ctx;
    CHECK_RC(activate(ctx));
    if (!rebuild) return neighbors_refresh(ctx, &s->nb);
    CHECK_RC(neighbors_sync_positions(ctx, &s->nb));
    int64_t P = 0;
    CHECK_RC(neighbors_build(ctx, &s->nb, 1, -1, &P, false));
    return TGAP_OK;
}

static int site_set(tgap_system *s, int central_species, SiteSet **out)
{
    for (auto &ss : s->site_sets)
        if (ss.central_species == central_species) {
            *out = &ss;
            return TGAP_OK;
        }
    tgap_context *ctx = s->ctx;
    std::vector<int> rows;
    const int beg = s->range_beg, end = s->range_end < 0 ? (int)s->host_species.size() : s->range_end;
    for (int i = beg; i < end; ++i)
        if (central_species == 0 || s->host_species[i] == central_species) rows.push_back(i);
    s->site_sets.emplace_back();
    SiteSet &ss = s->site_sets.back();
    ss.central_species = central_species;
    ss.n_rows = (int)rows.size();
    CHECK_RC(upload(ctx, ss.sites, rows.data(), rows.size()));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *out = &ss;
    return TGAP_OK;
}

static int ensure_eval_buffers(tgap_system *s, const tgap_model *m, int n_rows, int precision)
{
    const SoapParams &P = m->soap.p;
    const int nlm = (P.l_max + 1) * (P.l_max + 1);
    const size_t tsz = precision == TGAP_FP64 ? 8 : 4;
    const int q_ld = precision == TGAP_FP64 ? P.dim : m->gap.dim_pad;
    const int rows_pad = (n_rows + 127) / 128 * 128;
    if (s->c.ensure(tsz * (size_t)n_rows * P.n_max * nlm) || s->q.ensure(tsz * (size_t)rows_pad * q_ld) ||
        s->norm.ensure(tsz * (size_t)n_rows))
        return set_error(s->ctx, TGAP_ERR_NOMEM, "descriptor workspace");
    if (precision != TGAP_FP64) {
        const uint64_t e0 = g_alloc_epoch.load();
        if (s->q_hi.ensure(2 * (size_t)rows_pad * q_ld) || s->q_lo.ensure(2 * (size_t)rows_pad * q_ld))
            return set_error(s->ctx, TGAP_ERR_NOMEM, "descriptor workspace");
        // rows past n_rows feed the 128-row GEMM tiles: keep them zero (fresh buffers only)
        if (g_alloc_epoch.load() != e0) {
            TGAP_CUDA(s->ctx, cudaMemsetAsync(s->q_hi.ptr, 0, s->q_hi.bytes, s->ctx->stream));
            TGAP_CUDA(s->ctx, cudaMemsetAsync(s->q_lo.ptr, 0, s->q_lo.bytes, s->ctx->stream));
        }
    }
    return TGAP_OK;
}

// geom: the descriptor forward writes this step's pair geometry from the primitive positions
// (pure-replica systems; every site of the list must belong to some model's site set)
// queue: two zeroed site counters (forward, adjoint) for the persistent descriptor launches, or null
static int compute_model(tgap_context *ctx, tgap_system *s, const tgap_model *m, int precision,
                         int do_forces, double *d_energies, double *d_forces, double *d_virial, bool geom = false,
                         int *queue = nullptr)
{
    SiteSet *ss = nullptr;
    CHECK_RC(site_set(s, m->central_species, &ss));
    const int n_rows = ss->n_rows;
    if (n_rows == 0) return TGAP_OK;
    CHECK_RC(ensure_eval_buffers(s, m, n_rows, precision));
    PairView pv{s->nb.start.as<int64_t>(), s->nb.xyz.as<double>(), s->nb.rjs.as<double>(),
                s->nb.nspecies.as<int>(), s->nb.jatom.as<int>(), s->nb.n_atoms, ctx->d_check};
    PairView pvf = pv;  // the forward's view, writing the geometry first when asked
    if (queue) {
        pvf.queue = queue;
        pv.queue = queue + 1;
    }
    if (geom) {
        pvf.geo.pos = s->nb.positions.as<double>();
        pvf.geo.list = s->nb.list.as<int>();
        pvf.geo.site_struct = s->nb.site_struct.as<int>();
        pvf.geo.sd = s->nb.d_structs.ptr;
        pvf.geo.rjs_out = s->nb.rjs.as<double>();
        pvf.geo.xyz_out = s->nb.xyz.as<double>();
    }
    SoapOut o;
    o.c = s->c.ptr;
    o.q = s->q.ptr;
    o.norm = s->norm.ptr;
    const int *sites = ss->sites.as<int>();
    if (precision == TGAP_FP64) {
        o.q_ld = m->gap.dim;
        CHECK_RC(soap_forward(ctx, m->soap, pvf, sites, n_rows, TGAP_FP64, o));
        CHECK_RC(gap_energy_grad_f64(ctx, m->gap, (const double *)o.q, o.q_ld, n_rows, 0.0, do_forces,
                                     &s->gw, sites, nullptr, d_energies));
        if (do_forces)
            CHECK_RC(soap_backward(ctx, m->soap, pv, sites, n_rows, TGAP_FP64, o, s->gw.g.ptr, m->gap.dim,
                                   1, s->nb.site_struct.as<int>(), d_forces, d_virial));
    } else {
        if (!m->mixed_ready) return set_error(ctx, TGAP_ERR_UNSUPPORTED, "mixed path not prepared");
        o.q_ld = m->gap.dim_pad;
        o.q_hi = s->q_hi.as<__nv_bfloat16>();
        o.q_lo = s->q_lo.as<__nv_bfloat16>();
        // the fused GAP kernel accumulates dE/dq: the forward clears each row it writes
        const bool clear_g = do_forces && m->gap.dim_pad <= 384;
        if (clear_g) {
            const size_t rows_pad = ((size_t)n_rows + 127) / 128 * 128;
            if (s->gw.g.ensure(4 * rows_pad * m->gap.dim_pad)) return set_error(ctx, TGAP_ERR_NOMEM, "dE/dq rows");
            o.g_clear = s->gw.g.as<float>();
        }
        CHECK_RC(soap_forward(ctx, m->soap, pvf, sites, n_rows, TGAP_MIXED, o));
        CHECK_RC(gap_energy_grad_mixed(ctx, m->gap, o.q_hi, o.q_lo, n_rows, 0.0, do_forces, &s->gw, sites,
                                       nullptr, d_energies, nullptr, clear_g));
        if (do_forces)
            CHECK_RC(soap_backward(ctx, m->soap, pv, sites, n_rows, TGAP_MIXED, o, s->gw.g.ptr,
                                   m->gap.dim_pad, 0, s->nb.site_struct.as<int>(), d_forces, d_virial));
    }
    return TGAP_OK;
}

// zeroed: the caller cleared the outputs already (the MD step clears its contiguous block at once,
// with kQueueInts zeroed site counters at queue)
static int compute_models(tgap_context *ctx, tgap_system *s, int n_models, tgap_model *const *models,
                          int precision, int do_forces, double *d_energies, double *d_forces, double *d_virial,
                          bool geom, bool zeroed, int *queue = nullptr);

extern "C" int tgap_compute(tgap_context *ctx, tgap_system *s, int n_models, tgap_model *const *models,
                            int precision, int do_forces, double *d_energies, double *d_forces,
                            double *d_virial)
{
    return compute_models(ctx, s, n_models, models, precision, do_forces, d_energies, d_forces, d_virial, false,
                          false);
}

static int compute_models(tgap_context *ctx, tgap_system *s, int n_models, tgap_model *const *models,
                          int precision, int do_forces, double *d_energies, double *d_forces, double *d_virial,
                          bool geom, bool zeroed, int *queue)
{
    CHECK_RC(activate(ctx));
    if (!s || n_models <= 0 || !models || !d_energies || (do_forces && (!d_forces || !d_virial)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_compute: bad arguments");
    if (precision != TGAP_FP64 && precision != TGAP_MIXED)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "precision");
    const int N = s->nb.n_atoms;
    if (!zeroed) TGAP_CUDA(ctx, cudaMemsetAsync(d_energies, 0, sizeof(double) * N, ctx->stream));
    if (do_forces && !zeroed) {
        TGAP_CUDA(ctx, cudaMemsetAsync(d_forces, 0, sizeof(double) * 3 * N, ctx->stream));
        TGAP_CUDA(ctx, cudaMemsetAsync(d_virial, 0, sizeof(double) * 9 * s->nb.n_structures, ctx->stream));
    }
    if (!zeroed && 2 * n_models <= kQueueInts) {
        if (s->queue.ensure(sizeof(int) * kQueueInts)) return set_error(ctx, TGAP_ERR_NOMEM, "site counters");
        TGAP_CUDA(ctx, cudaMemsetAsync(s->queue.ptr, 0, sizeof(int) * kQueueInts, ctx->stream));
        queue = s->queue.as<int>();
    }
    if (2 * n_models > kQueueInts) queue = nullptr;
    for (int i = 0; i < n_models; ++i)
        CHECK_RC(compute_model(ctx, s, models[i], precision, do_forces, d_energies, d_forces, d_virial, geom,
                               queue ? queue + 2 * i : nullptr));
    if (!s->host_e0.empty()) {
        // turbogap_main.f90:994: the total energy of each atom adds its e0
        // the atoms of this system's site range only, so ranks that split the sites count each once
        const int beg = s->range_beg, end = s->range_end < 0 ? N : s->range_end;
        if (end > beg)
            k_add_e0<<<(end - beg + 255) / 256, 256, 0, ctx->stream>>>(beg, end, s->d_e0.as<double>(), d_energies);
        TGAP_LAUNCH_CHECK(ctx);
    }
    return TGAP_OK;
}

extern "C" int tgap_local_property(tgap_context *ctx, tgap_system *s, tgap_model *m, double V0, int precision,
                                   int do_derivatives, double *d_V, double *d_V_der)
{
    CHECK_RC(activate(ctx));
    if (!s || !m || !d_V || (do_derivatives && !d_V_der))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_local_property: bad arguments");
    if (precision != TGAP_FP64 && precision != TGAP_MIXED) return set_error(ctx, TGAP_ERR_ARGUMENT, "precision");
    const int N = s->nb.n_atoms;
    TGAP_CUDA(ctx, cudaMemsetAsync(d_V, 0, sizeof(double) * N, ctx->stream));
    if (do_derivatives) {
        CHECK_RC(neighbors_sync_count(ctx, &s->nb));
        TGAP_CUDA(ctx, cudaMemsetAsync(d_V_der, 0, sizeof(double) * 3 * (size_t)s->nb.n_pairs, ctx->stream));
    }
    SiteSet *ss = nullptr;
    CHECK_RC(site_set(s, m->central_species, &ss));
    const int n_rows = ss->n_rows;
    if (n_rows == 0) return TGAP_OK;
    CHECK_RC(ensure_eval_buffers(s, m, n_rows, precision));
    DeviceModel gm = m->gap;  // shallow copy: the same device operands, the local-property zeta test
    gm.zeta_tol = 1.0e-10;
    gm.zeta_nint = true;
    PairView pv{s->nb.start.as<int64_t>(), s->nb.xyz.as<double>(), s->nb.rjs.as<double>(),
                s->nb.nspecies.as<int>(), s->nb.jatom.as<int>(), s->nb.n_atoms, ctx->d_check};
    SoapOut o;
    o.c = s->c.ptr;
    o.q = s->q.ptr;
    o.norm = s->norm.ptr;
    const int *sites = ss->sites.as<int>();
    const void *g = nullptr;
    int g_ld = 0, g_double = 0;
    if (precision == TGAP_FP64) {
        o.q_ld = m->gap.dim;
        CHECK_RC(soap_forward(ctx, m->soap, pv, sites, n_rows, TGAP_FP64, o));
        CHECK_RC(gap_energy_grad_f64(ctx, gm, (const double *)o.q, o.q_ld, n_rows, V0, do_derivatives, &s->gw, sites,
                                     nullptr, d_V));
        g = s->gw.g.ptr;
        g_ld = m->gap.dim;
        g_double = 1;
    } else {
        if (!m->mixed_ready) return set_error(ctx, TGAP_ERR_UNSUPPORTED, "mixed path not prepared");
        o.q_ld = m->gap.dim_pad;
        o.q_hi = s->q_hi.as<__nv_bfloat16>();
        o.q_lo = s->q_lo.as<__nv_bfloat16>();
        CHECK_RC(soap_forward(ctx, m->soap, pv, sites, n_rows, TGAP_MIXED, o));
        CHECK_RC(gap_energy_grad_mixed(ctx, gm, o.q_hi, o.q_lo, n_rows, V0, do_derivatives, &s->gw, sites, nullptr,
                                       d_V));
        g = s->gw.g.ptr;
        g_ld = m->gap.dim_pad;
    }
    CHECK_RC(clip_nonneg(ctx, N, d_V));
    if (do_derivatives) {
        pv.pair_der = d_V_der;
        pv.gate = d_V;
        CHECK_RC(soap_backward(ctx, m->soap, pv, sites, n_rows, precision, o, g, g_ld, g_double, nullptr, nullptr,
                               nullptr));
    }
    return TGAP_OK;
}

// ============================================================================ autotuner

// Mean time of `stage` over the last timed runs (ms), or -1 when it did not run.
static double stage_mean_ms(tgap_context *ctx, const std::string &stage)
{
    timing_collect(ctx);
    for (size_t i = 0; i < ctx->stage_names.size(); ++i)
        if (ctx->stage_names[i] == stage && ctx->stage_count[i] > 0) return ctx->stage_ms[i] / ctx->stage_count[i];
    return -1.0;
}

extern "C" int tgap_autotune(tgap_context *ctx, tgap_system *s, int n_models, tgap_model *const *models,
                             int precision, int reps)
{
    graphs_stale();
    CHECK_RC(activate(ctx));
    if (!s || n_models <= 0 || !models || reps < 1) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_autotune: bad arguments");
    const int N = s->nb.n_atoms;
    DevBuf out;
    std::unique_ptr<DevBuf, void (*)(DevBuf *)> guard(&out, [](DevBuf *b) { b->release(); });
    if (out.ensure(sizeof(double) * (4 * (size_t)N + 9 * (size_t)s->nb.n_structures)))
        return set_error(ctx, TGAP_ERR_NOMEM, "autotuner outputs");
    double *d_e = out.as<double>(), *d_f = d_e + N, *d_v = d_f + 3 * (size_t)N;
    auto run = [&]() { return tgap_compute(ctx, s, n_models, models, precision, 1, d_e, d_f, d_v); };
    const bool timing0 = ctx->timing;
    timing_collect(ctx);
    const std::vector<double> ms0 = ctx->stage_ms;
    const std::vector<int64_t> cnt0 = ctx->stage_count;
    // discovery: the launches of this evaluation register their keys
    ctx->probe_key.clear();
    ctx->tune_seen.clear();
    int rc = run();
    const auto seen = ctx->tune_seen;
    std::string report;
    for (const auto &kv : seen) {
        if (rc) break;
        const std::string &key = kv.first;
        const tgap_context::TuneSlot &slot = kv.second;
        int best = slot.dflt;
        double best_ms = -1.0, dflt_ms = -1.0;
        for (int cand : slot.candidates) {
            ctx->probe_key = key;
            ctx->probe_val = cand;
            ctx->timing = false;
            if ((rc = run())) break;  // warm-up (first launch of a variant sets its attributes)
            timing_collect(ctx);
            for (auto &v : ctx->stage_ms) v = 0.0;
            for (auto &c : ctx->stage_count) c = 0;
            ctx->timing = true;
            for (int r = 0; r < reps && !rc; ++r) rc = run();
            ctx->timing = false;
            if (rc) break;
            const double ms = stage_mean_ms(ctx, slot.stage);
            if (cand == slot.dflt) dflt_ms = ms;
            if (ms >= 0.0 && (best_ms < 0.0 || ms < best_ms)) {
                best_ms = ms;
                best = cand;
            }
        }
        ctx->probe_key.clear();
        if (rc) break;
        ctx->tune[key] = best;
        char line[256];
        std::snprintf(line, sizeof(line), "%s %d %.2f us (default %d: %.2f us)\n", key.c_str(), best, 1e3 * best_ms,
                      slot.dflt, 1e3 * dflt_ms);
        report += line;
    }
    ctx->probe_key.clear();
    // the caller's stage timers as they were
    timing_collect(ctx);
    for (size_t i = 0; i < ctx->stage_ms.size(); ++i) {
        ctx->stage_ms[i] = i < ms0.size() ? ms0[i] : 0.0;
        ctx->stage_count[i] = i < cnt0.size() ? cnt0[i] : 0;
    }
    ctx->timing = timing0;
    if (rc) return rc;
    ctx->tune_report = report;
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return read_device_check(ctx);
}

extern "C" int tgap_autotune_report(tgap_context *ctx, char *buf, int64_t cap, int64_t *needed)
{
    if (!ctx) return TGAP_ERR_ARGUMENT;
    const int64_t n = (int64_t)ctx->tune_report.size() + 1;
    if (needed) *needed = n;
    if (!buf || cap < n) return buf ? TGAP_ERR_CAPACITY : TGAP_OK;
    std::memcpy(buf, ctx->tune_report.c_str(), (size_t)n);
    return TGAP_OK;
}

extern "C" int tgap_autotune_clear(tgap_context *ctx)
{
    graphs_stale();
    if (!ctx) return TGAP_ERR_ARGUMENT;
    ctx->tune.clear();
    ctx->tune_suffix.clear();
    ctx->tune_report.clear();
    return TGAP_OK;
}

extern "C" int tgap_autotune_set(tgap_context *ctx, const char *key, int value)
{
    graphs_stale();
    if (!ctx || !key || !key[0]) return TGAP_ERR_ARGUMENT;
    if (key[0] == '*') {
        const std::string suffix(key + 1);
        for (auto &pat : ctx->tune_suffix)
            if (pat.first == suffix) {
                pat.second = value;
                return TGAP_OK;
            }
        ctx->tune_suffix.emplace_back(suffix, value);
    } else {
        ctx->tune[key] = value;
    }
    return TGAP_OK;
}

// The descriptor forward can write each step's pair geometry itself (compute_model's geom) on a
// pure-replica system whose every site belongs to some model's site set.
static bool can_fuse_geometry(const tgap_system *s, int n_models, const tgap_model *const *models)
{
    if (!s->nb.replicated) return false;
    std::vector<int> covered;
    for (int i = 0; i < n_models; ++i) {
        if (models[i]->central_species == 0) return true;
        covered.push_back(models[i]->central_species);
    }
    for (int sp : s->host_species)
        if (std::find(covered.begin(), covered.end(), sp) == covered.end()) return false;
    return true;
}

// One call of the host-buffer entry. A rebuild of existing lists runs on the device (no host
// synchronization before the forces); the pair count comes back with the results, and a list that
// outgrew the reserved arrays is rebuilt on the host and the call repeated (device_rebuild false).
// Without a rebuild the forward writes the pair geometry itself where it can.
static int calculate_gap_soap(tgap_context *ctx, tgap_system *s, int n_models, tgap_model *const *models,
                              int precision, const double *positions, int rebuild, bool device_rebuild,
                              double *energies, double *forces, double *virial)
{
    const int N = s->nb.n_atoms, nst = s->nb.n_structures;
    const size_t out_bytes = sizeof(double) * ((size_t)N + 3 * (size_t)N + 9 * (size_t)nst);
    if (ctx->pinned[0].ensure(sizeof(double) * 3 * (size_t)N) || ctx->pinned[1].ensure(out_bytes + 16) ||
        s->scratch_forces.ensure(out_bytes) || s->queue.ensure(sizeof(int) * kQueueInts))
        return set_error(ctx, TGAP_ERR_NOMEM, "staging buffers");
    if (n_models <= 0 || !models) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_calculate_gap_soap: bad model list");
    for (int i = 0; i < n_models; ++i)
        if (!models[i]) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_calculate_gap_soap: null model");
    // registered caller arrays are read and written directly, others through the staging buffers;
    // either way by a copy kernel over their device addresses
    void *in_dev = positions ? host_registered(ctx, positions, sizeof(double) * 3 * (size_t)N) : nullptr;
    void *out_dev[3] = {host_registered(ctx, energies, sizeof(double) * N),
                        forces ? host_registered(ctx, forces, sizeof(double) * 3 * (size_t)N) : nullptr,
                        virial ? host_registered(ctx, virial, sizeof(double) * 9 * (size_t)nst) : nullptr};
    const bool direct_in = in_dev != nullptr;
    const bool direct_out = out_dev[0] && (!forces || out_dev[1]) && (!virial || out_dev[2]);
    if (positions && !direct_in) {
        std::memcpy(ctx->pinned[0].ptr, positions, sizeof(double) * 3 * (size_t)N);
        in_dev = ctx->pinned[0].dev;
    }
    void *stage_dev = ctx->pinned[1].dev;  // the output staging buffer: energies, forces, virial, pair count
    if (!direct_out) {
        double *st = static_cast<double *>(stage_dev);
        out_dev[0] = st;
        out_dev[1] = st + N;
        out_dev[2] = st + 4 * (size_t)N;
    }
    const bool on_device = rebuild && device_rebuild && s->nb.list.ptr && s->nb.n_pairs > 0;
    const bool host_rebuild = rebuild && !on_device;
    const bool geom = !host_rebuild && can_fuse_geometry(s, n_models, models);
    const int do_forces = forces != nullptr || virial != nullptr;
    unsigned char *h = ctx->pinned[1].as<unsigned char>();
    // the device work of the call, stream-ordered; with a host rebuild (a host synchronization for
    // the pair count) it cannot be captured
    auto device_work = [&]() -> int {
        double *d_e = s->scratch_forces.as<double>();
        double *d_f = d_e + N;
        double *d_v = d_f + 3 * (size_t)N;
        // (more models than the counters cover: the descriptor launches without the work queue)
        const bool counters = 2 * n_models <= kQueueInts;
        {
            // the positions in; energies, forces and virial (one buffer) and the site counters cleared
            WordCopy in{};
            if (positions) {
                in.src[0] = static_cast<const unsigned long long *>(in_dev);
                in.dst[0] = s->nb.positions.as<unsigned long long>();
                in.n[0] = 3 * (long long)N;
            }
            in.zero[0] = reinterpret_cast<unsigned long long *>(d_e);
            in.nz[0] = (long long)(out_bytes / sizeof(unsigned long long));
            static_assert(kQueueInts % 2 == 0, "the site counters clear as 8-byte words");
            in.zero[1] = s->queue.as<unsigned long long>();
            in.nz[1] = counters ? kQueueInts / 2 : 0;
            CHECK_RC(copy_words(ctx, in));
        }
        if (on_device) {
            CHECK_RC(neighbors_sync_positions(ctx, &s->nb));
            CHECK_RC(neighbors_rebuild_lists_device(ctx, &s->nb, false));
            // the geometry comes from the forward where it can
            CHECK_RC(geom ? neighbors_maps(ctx, &s->nb) : neighbors_refresh(ctx, &s->nb));
        } else if (!geom) {
            CHECK_RC(tgap_system_update(s, host_rebuild ? 1 : 0));
        }
        CHECK_RC(compute_models(ctx, s, n_models, models, precision, do_forces, d_e, d_f, d_v, geom, true,
                                counters ? s->queue.as<int>() : nullptr));
        // energies, forces, virial and (after a rebuild) the unclamped pair count, in one launch
        WordCopy out{};
        const double *src[3] = {d_e, d_f, d_v};
        const long long len[3] = {N, forces ? 3 * (long long)N : 0, virial ? 9 * (long long)nst : 0};
        for (int a = 0; a < 3; ++a) {
            out.src[a] = reinterpret_cast<const unsigned long long *>(src[a]);
            out.dst[a] = static_cast<unsigned long long *>(out_dev[a]);
            out.n[a] = out_dev[a] ? len[a] : 0;
        }
        if (on_device) {
            out.src[3] = reinterpret_cast<const unsigned long long *>(s->nb.counts.as<int64_t>() + N);
            out.dst[3] = reinterpret_cast<unsigned long long *>(static_cast<unsigned char *>(stage_dev) + out_bytes);
            out.n[3] = 1;
        }
        CHECK_RC(copy_words(ctx, out));
        return TGAP_OK;
    };
    // A configuration (models, precision, rebuild on the device or not, geometry fused or not,
    // positions given, forces) runs eagerly the first time, which sizes every buffer, and from the
    // second time as one graph launch. Stage timing and per-launch checks keep the eager path.
    if (host_rebuild || ctx->timing || ctx->sync_check) {
        CHECK_RC(device_work());
    } else {
        const int flags = (on_device ? 1 : 0) | (geom ? 2 : 0) | (positions ? 4 : 0) | (do_forces ? 8 : 0) |
                          (direct_in ? 16 : 0) | (direct_out ? 32 : 0);
        // the caller's arrays are part of a graph that copies to or from them directly
        const void *io[4] = {direct_in ? positions : nullptr, direct_out ? energies : nullptr,
                             direct_out ? forces : nullptr, direct_out ? virial : nullptr};
        tgap_system::CallGraph *cg = nullptr;
        for (auto &c : s->call_graphs)
            if (c.precision == precision && c.flags == flags && (int)c.models.size() == n_models &&
                std::equal(c.models.begin(), c.models.end(), models) && std::equal(io, io + 4, c.io))
                cg = &c;
        if (!cg) {
            s->call_graphs.emplace_back();
            cg = &s->call_graphs.back();
            cg->models.assign(models, models + n_models);
            cg->precision = precision;
            cg->flags = flags;
            std::copy(io, io + 4, cg->io);
        }
        const uint64_t e0 = g_alloc_epoch.load(std::memory_order_relaxed);
        if (cg->epoch != e0) {
            // something the graph baked in changed (or nothing was captured yet): run eagerly once
            // more, which rebuilds host-side state such as site sets, before capturing again
            if (cg->exec) cudaGraphExecDestroy(cg->exec);
            if (cg->graph) cudaGraphDestroy(cg->graph);
            cg->exec = nullptr;
            cg->graph = nullptr;
            if (cg->seen && cg->seen_epoch != e0) cg->seen = false;
        }
        if (!cg->exec && cg->seen) {
            TGAP_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
            const int64_t launches = ctx->launches;
            int rc = device_work();
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
            cg->kernels = ctx->launches - launches;
            ctx->launches = launches;
            if (rc || ce != cudaSuccess || g_alloc_epoch.load(std::memory_order_relaxed) != e0) {
                if (g) cudaGraphDestroy(g);
                if (rc) return rc;
                if (ce != cudaSuccess) return cuda_check(ctx, ce, "call graph capture");
            } else {
                cg->graph = g;
                TGAP_CUDA(ctx, cudaGraphInstantiate(&cg->exec, g, 0));
                cg->epoch = e0;
            }
        }
        if (cg->exec) {
            TGAP_CUDA(ctx, cudaGraphLaunch(cg->exec, ctx->stream));
            ctx->launches += cg->kernels;
        } else {
            CHECK_RC(device_work());
            cg->seen = true;
            cg->seen_epoch = g_alloc_epoch.load(std::memory_order_relaxed);
        }
    }
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (on_device) {
        int64_t total = 0;
        std::memcpy(&total, h + out_bytes, sizeof(int64_t));
        s->nb.n_pairs = total;
        s->nb.count_on_device = false;
        if (total > s->nb.pair_capacity()) {
            // the device lists were clamped (and this call's results cut short): rebuild on the
            // host and repeat
            return calculate_gap_soap(ctx, s, n_models, models, precision, nullptr, 1, false, energies, forces,
                                      virial);
        }
    }
    if (!direct_out) {
        const double *hv = reinterpret_cast<const double *>(h);
        std::memcpy(energies, hv, sizeof(double) * N);
        if (forces) std::memcpy(forces, hv + N, sizeof(double) * 3 * (size_t)N);
        if (virial) std::memcpy(virial, hv + 4 * (size_t)N, sizeof(double) * 9 * (size_t)nst);
    }
    return TGAP_OK;
}

extern "C" int tgap_calculate_gap_soap(tgap_context *ctx, tgap_system *s, int n_models, tgap_model *const *models,
                                       int precision, const double *positions, int rebuild, double *energies,
                                       double *forces, double *virial)
{
    CHECK_RC(activate(ctx));
    if (!s || !energies) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_calculate_gap_soap: bad arguments");
    return calculate_gap_soap(ctx, s, n_models, models, precision, positions, rebuild, true, energies, forces,
                              virial);
}

extern "C" int tgap_descriptors(tgap_context *ctx, tgap_system *s, const tgap_model *m, int precision,
                                double *d_soap, int *n_rows)
{
    CHECK_RC(activate(ctx));
    if (!s || !m || !d_soap || !n_rows) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_descriptors");
    SiteSet *ss = nullptr;
    CHECK_RC(site_set(s, m->central_species, &ss));
    *n_rows = ss->n_rows;
    if (ss->n_rows == 0) return TGAP_OK;
    CHECK_RC(ensure_eval_buffers(s, m, ss->n_rows, TGAP_FP64));
    PairView pv{s->nb.start.as<int64_t>(), s->nb.xyz.as<double>(), s->nb.rjs.as<double>(),
                s->nb.nspecies.as<int>(), s->nb.jatom.as<int>(), s->nb.n_atoms, ctx->d_check};
    SoapOut o;
    o.c = s->c.ptr;
    o.q = d_soap;
    o.norm = s->norm.ptr;
    o.q_ld = m->gap.dim;
    (void)precision;
    return soap_forward(ctx, m->soap, pv, ss->sites.as<int>(), ss->n_rows, TGAP_FP64, o);
}

// ---------------------------------------------------------------------------- get_gap_soap

extern "C" int tgap_get_gap_soap(tgap_context *ctx, const tgap_soap_hypers *hypers, int n_total_sites,
                                 int n_sites0, const int *n_neigh0, const int *neighbors_list0,
                                 const double *rjs0, const double *xyz0, const int *species_supercell,
                                 int central_species, int n_sparse, const double *alphas, const double *Qs,
                                 double delta, double zeta, int do_forces, int precision,
                                 double *energies0, double *forces0, double *virial, double *soap_out)
{
    CHECK_RC(activate(ctx));
    if (!hypers || n_total_sites <= 0 || n_sites0 < 0 || !n_neigh0 || !neighbors_list0 || !rjs0 || !xyz0 ||
        !species_supercell || !alphas || !Qs || !energies0 || (do_forces && (!forces0 || !virial)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_get_gap_soap: bad arguments");
    tgap_model *m = nullptr;
    CHECK_RC(tgap_model_create(ctx, hypers, central_species, n_sparse, alphas, Qs, delta, zeta, &m));
    std::unique_ptr<tgap_model, int (*)(tgap_model *)> gm(m, tgap_model_destroy);
    // host-side pair view of the caller's list (gap_interface.f90:184-289 folds neighbors with
    // mod(j-1, n_total_sites)+1 and keeps pairs within rcut of known species)
    std::vector<int64_t> start(n_sites0 + 1, 0);
    for (int i = 0; i < n_sites0; ++i) start[i + 1] = start[i] + n_neigh0[i];
    const size_t P = (size_t)start[n_sites0];
    std::vector<int> sp(P), jat(P), rows;
    std::vector<unsigned char> seen(n_total_sites, 0);
    const double rcut_max = m->soap.p.rcut_max;
    for (int i = 0; i < n_sites0; ++i) {
        const int self = (neighbors_list0[start[i]] - 1) % n_total_sites;
        const int si = species_supercell[neighbors_list0[start[i]] - 1];
        const bool keep = central_species == 0 || si == central_species;
        if (keep) rows.push_back(i);
        for (int64_t k = start[i]; k < start[i + 1]; ++k) {
            const int j = neighbors_list0[k] - 1;
            sp[k] = species_supercell[j];
            jat[k] = j % n_total_sites;
            if (keep && rjs0[k] < rcut_max && sp[k] > 0) seen[jat[k]] = 1;
        }
        (void)self;
    }
    DevBuf *S = ctx->scratch;
    CHECK_RC(upload(ctx, S[10], start.data(), start.size()));
    CHECK_RC(upload(ctx, S[11], xyz0, 3 * P));
    CHECK_RC(upload(ctx, S[12], rjs0, P));
    CHECK_RC(upload(ctx, S[13], sp.data(), P));
    CHECK_RC(upload(ctx, S[14], jat.data(), P));
    CHECK_RC(upload(ctx, S[15], rows.data(), rows.size()));
    const int n_rows = (int)rows.size();
    const SoapParams &Pp = m->soap.p;
    const int nlm = (Pp.l_max + 1) * (Pp.l_max + 1);
    const int q_ld = precision == TGAP_FP64 ? Pp.dim : m->gap.dim_pad;
    const int rows_pad = (n_rows + 127) / 128 * 128;
    if (S[16].ensure(8 * (size_t)n_rows * Pp.n_max * nlm + 8) || S[17].ensure(8 * (size_t)rows_pad * q_ld + 8) ||
        S[18].ensure(8 * (size_t)n_rows + 8) || S[19].ensure(8 * (size_t)n_total_sites) ||
        S[20].ensure(8 * 3 * (size_t)n_total_sites) || S[21].ensure(8 * 9) ||
        S[22].ensure(2 * (size_t)rows_pad * q_ld + 8) || S[23].ensure(2 * (size_t)rows_pad * q_ld + 8))
        return set_error(ctx, TGAP_ERR_NOMEM, "get_gap_soap workspace");
    if (precision != TGAP_FP64) {
        TGAP_CUDA(ctx, cudaMemsetAsync(S[22].ptr, 0, 2 * (size_t)rows_pad * q_ld, ctx->stream));
        TGAP_CUDA(ctx, cudaMemsetAsync(S[23].ptr, 0, 2 * (size_t)rows_pad * q_ld, ctx->stream));
    }
    PairView pv{S[10].as<int64_t>(), S[11].as<double>(), S[12].as<double>(), S[13].as<int>(), S[14].as<int>(),
                n_total_sites, ctx->d_check};
    SoapOut o;
    o.c = S[16].ptr;
    o.q = S[17].ptr;
    o.norm = S[18].ptr;
    o.q_ld = q_ld;
    double *d_e = S[19].as<double>(), *d_f = S[20].as<double>(), *d_v = S[21].as<double>();
    TGAP_CUDA(ctx, cudaMemsetAsync(d_e, 0, 8 * (size_t)n_total_sites, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(d_f, 0, 8 * 3 * (size_t)n_total_sites, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(d_v, 0, 8 * 9, ctx->stream));
    GapWork w;
    int rc = TGAP_OK;
    // the kernels index sites by position in the caller's list; rows map to atoms via jatom of
    // the self slot, so energies/forces land on folded global indices
    std::vector<int> row_atom(n_rows);
    for (int r = 0; r < n_rows; ++r) row_atom[r] = jat[start[rows[r]]];
    CHECK_RC(upload(ctx, S[9], row_atom.data(), row_atom.size()));
    if (precision == TGAP_FP64) {
        rc = soap_forward(ctx, m->soap, pv, S[15].as<int>(), n_rows, TGAP_FP64, o);
        if (!rc) rc = gap_energy_grad_f64(ctx, m->gap, (const double *)o.q, q_ld, n_rows, 0.0, do_forces, &w,
                                          S[9].as<int>(), nullptr, d_e);
        if (!rc && do_forces)
            rc = soap_backward(ctx, m->soap, pv, S[15].as<int>(), n_rows, TGAP_FP64, o, w.g.ptr, Pp.dim, 1,
                               nullptr, d_f, d_v);
    } else {
        o.q_hi = S[22].as<__nv_bfloat16>();
        o.q_lo = S[23].as<__nv_bfloat16>();
        rc = soap_forward(ctx, m->soap, pv, S[15].as<int>(), n_rows, TGAP_MIXED, o);
        if (!rc) rc = gap_energy_grad_mixed(ctx, m->gap, o.q_hi, o.q_lo, n_rows, 0.0, do_forces, &w,
                                            S[9].as<int>(), nullptr, d_e);
        if (!rc && do_forces)
            rc = soap_backward(ctx, m->soap, pv, S[15].as<int>(), n_rows, TGAP_MIXED, o, w.g.ptr, m->gap.dim_pad,
                               0, nullptr, d_f, d_v);
    }
    std::vector<double> he(n_total_sites), hf(3 * (size_t)n_total_sites);
    if (!rc) rc = download(ctx, he.data(), S[19], (size_t)n_total_sites);
    if (!rc && do_forces) rc = download(ctx, hf.data(), S[20], 3 * (size_t)n_total_sites);
    if (!rc && do_forces) rc = download(ctx, virial, S[21], 9);
    if (!rc && soap_out && precision == TGAP_FP64) {
        std::vector<double> q((size_t)n_rows * Pp.dim);
        rc = download(ctx, q.data(), S[17], q.size());
        if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = TGAP_ERR_CUDA;
        for (int r = 0; r < n_rows && !rc; ++r)
            std::memcpy(soap_out + (size_t)rows[r] * Pp.dim, q.data() + (size_t)r * Pp.dim, 8 * Pp.dim);
    }
    if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = TGAP_ERR_CUDA;
    if (!rc) {
        for (int r = 0; r < n_rows; ++r) energies0[row_atom[r]] = he[row_atom[r]];
        if (do_forces)
            for (int a = 0; a < n_total_sites; ++a)
                if (seen[a])
                    for (int x = 0; x < 3; ++x) forces0[3 * (size_t)a + x] = hf[3 * (size_t)a + x];
    }
    DevBuf *wb[] = {&w.e_part, &w.G, &w.g, &w.G_hi, &w.G_lo};
    for (DevBuf *b : wb) b->release();
    return rc;
}

// ============================================================================ MD

struct tgap_terms {
    tgap_context *ctx;
    TermSet set;
};

struct tgap_md {
    tgap_context *ctx;
    tgap_system *sys;
    std::vector<tgap_model *> models;
    tgap_terms *terms = nullptr;  // pair and triplet terms added after the SOAP models
    DevBuf out;  // forces (3 N), energies (N), virial (9 per structure), site counters: one clear per step
    int *queue = nullptr;  // the site counters in out (kQueueInts)
    // the descriptor forward writes each step's pair geometry (no separate geometry pass): a
    // pure-replica system whose sites all belong to some model, and no pair/triplet terms
    bool fused_geom = false;
    int precision, rebuild_every, use_graph;
    double dt, dt_prev = 0.0;
    int64_t step = 0;
    bool first = true;
    DevBuf mass, vel, forces, forces_prev, pos_prev, energies, virial;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t graph_epoch = 0;  // allocation epoch the graph was captured at
    int64_t graph_kernels = 0;
    // the steps between two list rebuilds (rebuild_every - 1 of them) as one graph
    cudaGraph_t graph_run = nullptr;
    cudaGraphExec_t exec_run = nullptr;
    uint64_t run_epoch = 0;
    int64_t run_kernels = 0;
    // list rebuilds after the first run on the device inside the step graphs, with no read-back
    // of the pair count (neighbors_rebuild_lists_device): systems without pair/triplet terms,
    // whose buffers follow the host count
    bool device_rebuild = false;
    uint64_t settled_epoch = 0;  // graph epoch at the last eager step (graphs are captured only at it)
    // a whole rebuild cycle (the rebuild step and the rebuild_every - 1 steps after it) as one graph
    cudaGraph_t graph_cycle = nullptr;
    cudaGraphExec_t exec_cycle = nullptr;
    uint64_t cycle_epoch = 0;
    int64_t cycle_kernels = 0;
    // one rebuild step as a graph (when fewer steps than a cycle are asked for)
    cudaGraph_t graph_rb = nullptr;
    cudaGraphExec_t exec_rb = nullptr;
    uint64_t rb_epoch = 0;
    int64_t rb_kernels = 0;
};

static int terms_add(tgap_context *ctx, tgap_system *s, tgap_terms *t, int do_forces, double *d_e, double *d_f,
                     double *d_v)
{
    if (t->set.rcut_max() > s->rcut)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "terms reach %g A, beyond the system's list cutoff %g A",
                         t->set.rcut_max(), s->rcut);
    if (!s->d_species.ptr) CHECK_RC(upload(ctx, s->d_species, s->host_species.data(), s->host_species.size()));
    NeighborBatch &nb = s->nb;
    return terms_compute(ctx, t->set, nb.n_atoms, nb.start.as<int64_t>(), nb.rjs.as<double>(), nb.xyz.as<double>(),
                         s->d_species.as<int>(), nb.nspecies.as<int>(), nb.jatom.as<int>(), nb.site_struct.as<int>(),
                         do_forces, d_e, d_f, d_v);
}

static bool md_can_fuse_geometry(const tgap_md *md)
{
    return !md->terms && can_fuse_geometry(md->sys, (int)md->models.size(), md->models.data());
}

static int md_eval(tgap_md *md)
{
    TGAP_CUDA(md->ctx, cudaMemsetAsync(md->out.ptr, 0, md->out.bytes, md->ctx->stream));
    CHECK_RC(compute_models(md->ctx, md->sys, (int)md->models.size(), md->models.data(), md->precision, 1,
                            md->energies.as<double>(), md->forces.as<double>(), md->virial.as<double>(),
                            md->fused_geom, true, md->queue));
    if (md->terms)
        CHECK_RC(terms_add(md->ctx, md->sys, md->terms, 1, md->energies.as<double>(), md->forces.as<double>(),
                           md->virial.as<double>()));
    return TGAP_OK;
}

// one step after the first: geometry refresh, forces, velocity Verlet; with rebuild, new lists on
// this step's positions first, built on the device (the refresh gives them their species, atom
// maps and geometry)
static int md_step_body(tgap_md *md, bool rebuild = false)
{
    tgap_context *ctx = md->ctx;
    if (rebuild) {
        CHECK_RC(neighbors_sync_positions(ctx, &md->sys->nb));
        CHECK_RC(neighbors_rebuild_lists_device(ctx, &md->sys->nb, true));
        // the new lists' species and atom maps; their geometry comes from the forward when fused
        CHECK_RC(md->fused_geom ? neighbors_maps(ctx, &md->sys->nb) : neighbors_refresh(ctx, &md->sys->nb));
    } else if (!md->fused_geom) {
        CHECK_RC(neighbors_refresh(ctx, &md->sys->nb));
    }
    CHECK_RC(md_eval(md));
    CHECK_RC(velocity_verlet(ctx, md->sys->nb.n_atoms, md->sys->nb.positions.as<double>(),
                             md->pos_prev.as<double>(), md->vel.as<double>(), md->forces.as<double>(),
                             md->forces_prev.as<double>(), md->mass.as<double>(), md->dt, md->dt, 0));
    return TGAP_OK;
}

// ---------------------------------------------------------------------------- pair/triplet terms

extern "C" int tgap_terms_create(tgap_context *ctx, tgap_terms **out)
{
    if (!ctx || !out) return TGAP_ERR_ARGUMENT;
    auto *t = new tgap_terms();
    t->ctx = ctx;
    *out = t;
    return TGAP_OK;
}

extern "C" int tgap_terms_destroy(tgap_terms *t)
{
    if (!t) return TGAP_OK;
    cudaSetDevice(t->ctx->device);
    cudaStreamSynchronize(t->ctx->stream);
    t->set.release();
    delete t;
    return TGAP_OK;
}

extern "C" int tgap_terms_add_2b(tgap_terms *t, int species1, int species2, int n_sparse, const double *alphas,
                                 const double *cutoff, const double *Qs, double rcut, double buffer, double delta,
                                 double sigma, double e0)
{
    if (!t) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = t->ctx;
    CHECK_RC(activate(ctx));
    if (n_sparse < 1 || !alphas || !cutoff || !Qs || !(rcut > 0) || !(buffer > 0) || !(sigma > 0))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_terms_add_2b: bad arguments");
    Term2b b;
    b.sp1 = species1;
    b.sp2 = species2;
    b.n_sparse = n_sparse;
    b.rcut = rcut;
    b.buffer = buffer;
    b.delta = delta;
    b.sigma = sigma;
    b.e0 = e0;
    int rc = upload(ctx, b.alphas, alphas, (size_t)n_sparse);
    if (!rc) rc = upload(ctx, b.cutoff, cutoff, (size_t)n_sparse);
    if (!rc) rc = upload(ctx, b.Qs, Qs, (size_t)n_sparse);
    if (rc) {
        for (DevBuf *p : {&b.alphas, &b.cutoff, &b.Qs}) p->release();
        return rc;
    }
    t->set.t2b.push_back(b);
    return TGAP_OK;
}

extern "C" int tgap_terms_add_core_pot(tgap_terms *t, int species1, int species2, int n, const double *x,
                                       const double *V, double yp1, double ypn, const double *dVdx2)
{
    if (!t) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = t->ctx;
    CHECK_RC(activate(ctx));
    if (n < 2 || !x || !V || !dVdx2) return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_terms_add_core_pot: bad arguments");
    TermCore c;
    c.sp1 = species1;
    c.sp2 = species2;
    c.n = n;
    c.yp1 = yp1;
    c.ypn = ypn;
    c.rcut = x[0];
    for (int i = 1; i < n; ++i) {
        if (!(x[i] > x[i - 1]))  // splines.f90 stops on h = 0
            return set_error(ctx, TGAP_ERR_ARGUMENT, "core_pot table: x must increase (x[%d] <= x[%d])", i, i - 1);
        c.rcut = std::max(c.rcut, x[i]);
    }
    int rc = upload(ctx, c.x, x, (size_t)n);
    if (!rc) rc = upload(ctx, c.V, V, (size_t)n);
    if (!rc) rc = upload(ctx, c.y2, dVdx2, (size_t)n);
    if (rc) {
        for (DevBuf *p : {&c.x, &c.V, &c.y2}) p->release();
        return rc;
    }
    t->set.core.push_back(c);
    return TGAP_OK;
}

extern "C" int tgap_terms_add_3b(tgap_terms *t, int species_center, int species1, int species2, int n_sparse,
                                 const double *alphas, const double *cutoff, const double *Qs, double rcut,
                                 double buffer, double delta, const double *sigma, double e0, int kernel_type)
{
    if (!t) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = t->ctx;
    CHECK_RC(activate(ctx));
    if (n_sparse < 1 || !alphas || !cutoff || !Qs || !sigma || !(rcut > 0) || !(buffer > 0) ||
        !(sigma[0] > 0 && sigma[1] > 0 && sigma[2] > 0) || (kernel_type != 0 && kernel_type != 1))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_terms_add_3b: bad arguments");
    Term3b b;
    b.sp0 = species_center;
    b.sp1 = species1;
    b.sp2 = species2;
    b.n_sparse = n_sparse;
    b.kernel = kernel_type;
    b.rcut = rcut;
    b.buffer = buffer;
    b.e0 = e0;
    for (int c = 0; c < 3; ++c) b.is[c] = 1.0 / (sigma[c] * sigma[c]);
    std::vector<double> pref(n_sparse);
    for (int s = 0; s < n_sparse; ++s) pref[s] = 2.0 * delta * delta * alphas[s] * cutoff[s];  // gap.f90:829
    int rc = upload(ctx, b.pref, pref.data(), pref.size());
    if (!rc) rc = upload(ctx, b.Qs, Qs, 3 * (size_t)n_sparse);
    if (rc) {
        for (DevBuf *p : {&b.pref, &b.Qs}) p->release();
        return rc;
    }
    t->set.t3b.push_back(b);
    return TGAP_OK;
}

extern "C" int tgap_terms_compute(tgap_context *ctx, tgap_system *s, tgap_terms *t, int do_forces, double *d_energies,
                                  double *d_forces, double *d_virial)
{
    CHECK_RC(activate(ctx));
    if (!s || !t || !d_energies || (do_forces && (!d_forces || !d_virial)))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_terms_compute: bad arguments");
    return terms_add(ctx, s, t, do_forces, d_energies, d_forces, d_virial);
}

extern "C" int tgap_md_set_terms(tgap_md *md, tgap_terms *t)
{
    if (!md) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = md->ctx;
    CHECK_RC(activate(ctx));
    if (t && t->set.rcut_max() > md->sys->rcut)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "terms reach %g A, beyond the system's list cutoff %g A",
                         t->set.rcut_max(), md->sys->rcut);
    if (t && !md->sys->d_species.ptr)
        CHECK_RC(upload(ctx, md->sys->d_species, md->sys->host_species.data(), md->sys->host_species.size()));
    md->terms = t;
    md->fused_geom = md_can_fuse_geometry(md);
    md->device_rebuild = !md->terms;
    // the step graphs change
    if (md->exec) cudaGraphExecDestroy(md->exec);
    if (md->graph) cudaGraphDestroy(md->graph);
    if (md->exec_run) cudaGraphExecDestroy(md->exec_run);
    if (md->graph_run) cudaGraphDestroy(md->graph_run);
    if (md->exec_cycle) cudaGraphExecDestroy(md->exec_cycle);
    if (md->graph_cycle) cudaGraphDestroy(md->graph_cycle);
    if (md->exec_rb) cudaGraphExecDestroy(md->exec_rb);
    if (md->graph_rb) cudaGraphDestroy(md->graph_rb);
    md->exec_rb = nullptr;
    md->graph_rb = nullptr;
    md->exec = nullptr;
    md->graph = nullptr;
    md->exec_run = nullptr;
    md->graph_run = nullptr;
    md->exec_cycle = nullptr;
    md->graph_cycle = nullptr;
    return TGAP_OK;
}

extern "C" int tgap_md_create(tgap_context *ctx, tgap_system *sys, int n_models, tgap_model *const *models,
                              const double *masses_amu, double dt, int rebuild_every, int precision,
                              int use_graph, tgap_md **out)
{
    CHECK_RC(activate(ctx));
    if (!sys || n_models <= 0 || !models || !masses_amu || !(dt > 0) || rebuild_every < 1 || !out)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_md_create: bad arguments");
    auto *md = new tgap_md();
    md->ctx = ctx;
    md->sys = sys;
    md->models.assign(models, models + n_models);
    md->precision = precision;
    md->fused_geom = md_can_fuse_geometry(md);
    md->device_rebuild = !md->terms;
    md->rebuild_every = rebuild_every;
    md->use_graph = use_graph;
    md->dt = dt;
    const int N = sys->nb.n_atoms;
    std::vector<double> m(N);
    for (int i = 0; i < N; ++i) m[i] = masses_amu[i] * 103.6426965268;  // read_files.f90:333
    int rc = upload(ctx, md->mass, m.data(), (size_t)N);
    DevBuf *bufs[] = {&md->vel, &md->forces_prev, &md->pos_prev};
    for (DevBuf *b : bufs)
        if (!rc && (b->ensure(sizeof(double) * 3 * N) || cudaMemsetAsync(b->ptr, 0, sizeof(double) * 3 * N, ctx->stream)))
            rc = TGAP_ERR_NOMEM;
    // forces, energies, virial and the site counters share one block (views into md->out, never
    // resized), cleared by one memset per step
    const size_t n_out = 4 * (size_t)N + 9 * (size_t)sys->nb.n_structures + kQueueInts / 2;
    if (!rc && (md->out.ensure(sizeof(double) * n_out) ||
                cudaMemsetAsync(md->out.ptr, 0, sizeof(double) * n_out, ctx->stream)))
        rc = TGAP_ERR_NOMEM;
    if (!rc) {
        double *o = md->out.as<double>();
        md->forces.ptr = o;
        md->forces.bytes = sizeof(double) * 3 * (size_t)N;
        md->energies.ptr = o + 3 * (size_t)N;
        md->energies.bytes = sizeof(double) * (size_t)N;
        md->virial.ptr = o + 4 * (size_t)N;
        md->virial.bytes = sizeof(double) * 9 * (size_t)sys->nb.n_structures;
        md->queue = reinterpret_cast<int *>(o + 4 * (size_t)N + 9 * (size_t)sys->nb.n_structures);
    }
    if (rc) {
        tgap_md_destroy(md);
        return rc;
    }
    *out = md;
    return TGAP_OK;
}

extern "C" int tgap_md_destroy(tgap_md *md)
{
    if (!md) return TGAP_OK;
    cudaSetDevice(md->ctx->device);
    if (md->exec) cudaGraphExecDestroy(md->exec);
    if (md->graph) cudaGraphDestroy(md->graph);
    if (md->exec_run) cudaGraphExecDestroy(md->exec_run);
    if (md->graph_run) cudaGraphDestroy(md->graph_run);
    if (md->exec_cycle) cudaGraphExecDestroy(md->exec_cycle);
    if (md->graph_cycle) cudaGraphDestroy(md->graph_cycle);
    if (md->exec_rb) cudaGraphExecDestroy(md->exec_rb);
    if (md->graph_rb) cudaGraphDestroy(md->graph_rb);
    DevBuf *bufs[] = {&md->mass, &md->vel, &md->forces_prev, &md->pos_prev, &md->out};
    for (DevBuf *b : bufs) b->release();
    delete md;
    return TGAP_OK;
}

extern "C" int tgap_md_set_velocities(tgap_md *md, const double *v)
{
    if (!md || !v) return TGAP_ERR_ARGUMENT;
    CHECK_RC(activate(md->ctx));
    TGAP_CUDA(md->ctx, cudaMemcpyAsync(md->vel.ptr, v, sizeof(double) * 3 * md->sys->nb.n_atoms,
                                       cudaMemcpyHostToDevice, md->ctx->stream));
    return TGAP_OK;
}

// Captures n_steps step bodies into one graph (re-captured when an allocation moved a buffer); the
// first of them rebuilds the lists on the device when rebuild_first is set.
static int md_graph(tgap_md *md, int n_steps, cudaGraph_t *graph, cudaGraphExec_t *exec, uint64_t *epoch,
                    int64_t *kernels, bool rebuild_first = false)
{
    tgap_context *ctx = md->ctx;
    if (*exec && *epoch == g_alloc_epoch.load(std::memory_order_relaxed)) return TGAP_OK;
    if (*exec) cudaGraphExecDestroy(*exec);
    if (*graph) cudaGraphDestroy(*graph);
    *exec = nullptr;
    *graph = nullptr;
    const uint64_t e0 = g_alloc_epoch.load(std::memory_order_relaxed);
    TGAP_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    const int64_t launches = ctx->launches;
    int rc = TGAP_OK;
    for (int i = 0; i < n_steps && !rc; ++i) rc = md_step_body(md, rebuild_first && i == 0);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
    *kernels = ctx->launches - launches;
    ctx->launches = launches;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) return cuda_check(ctx, ce, "graph capture");
    *graph = g;
    TGAP_CUDA(ctx, cudaGraphInstantiate(exec, g, 0));
    *epoch = e0;
    return TGAP_OK;
}

extern "C" int tgap_md_run(tgap_md *md, int n_steps)
{
    if (!md || n_steps < 0) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = md->ctx;
    CHECK_RC(activate(ctx));
    for (int it = 0; it < n_steps; ++it) {
        const bool rebuild = (md->step % md->rebuild_every) == 0;
        // after any change that makes the captured graphs stale, one step runs eagerly (it rebuilds
        // host-side state such as site sets, which cannot happen inside a capture) before graphs
        // are captured again
        const bool graphs = md->use_graph && !md->first &&
                            md->settled_epoch == g_alloc_epoch.load(std::memory_order_relaxed);
        // a whole rebuild cycle goes out as one graph launch when the lists are rebuilt on the device
        if (graphs && rebuild && md->device_rebuild && n_steps - it >= md->rebuild_every) {
            CHECK_RC(md_graph(md, md->rebuild_every, &md->graph_cycle, &md->exec_cycle, &md->cycle_epoch,
                              &md->cycle_kernels, true));
            TGAP_CUDA(ctx, cudaGraphLaunch(md->exec_cycle, ctx->stream));
            ctx->launches += md->cycle_kernels;
            md->sys->nb.count_on_device = true;  // set at capture only: every replay rebuilds
            md->step += md->rebuild_every;
            it += md->rebuild_every - 1;
            continue;
        }
        // a full run of rebuild-free steps goes out as one graph launch
        const int run = md->rebuild_every - 1;
        if (graphs && !rebuild && run > 1 && md->step % md->rebuild_every == 1 && n_steps - it >= run) {
            CHECK_RC(md_graph(md, run, &md->graph_run, &md->exec_run, &md->run_epoch, &md->run_kernels));
            TGAP_CUDA(ctx, cudaGraphLaunch(md->exec_run, ctx->stream));
            ctx->launches += md->run_kernels;
            md->step += run;
            it += run - 1;
            continue;
        }
        if (!md->first && rebuild && !md->device_rebuild) {
            // new pair lists on the current positions (one host synchronization for the pair
            // count); the step below refreshes the geometry on them like any other step
            CHECK_RC(neighbors_sync_positions(ctx, &md->sys->nb));
            int64_t n_pairs = 0;
            CHECK_RC(neighbors_rebuild_lists(ctx, &md->sys->nb, -1, &n_pairs));
            // the per-pair species and atom maps of the new lists (the step refreshes geometry)
            if (md->fused_geom) CHECK_RC(neighbors_refresh(ctx, &md->sys->nb));
        }
        if (md->first) {
            // eager first step: it sizes every buffer
            CHECK_RC(tgap_system_update(md->sys, rebuild ? 1 : 0));
            CHECK_RC(md_eval(md));
            CHECK_RC(velocity_verlet(ctx, md->sys->nb.n_atoms, md->sys->nb.positions.as<double>(),
                                     md->pos_prev.as<double>(), md->vel.as<double>(), md->forces.as<double>(),
                                     md->forces_prev.as<double>(), md->mass.as<double>(), md->dt, md->dt,
                                     md->first ? 1 : 0));
            md->first = false;
            md->settled_epoch = g_alloc_epoch.load(std::memory_order_relaxed);
        } else if (graphs && rebuild && md->device_rebuild) {
            CHECK_RC(md_graph(md, 1, &md->graph_rb, &md->exec_rb, &md->rb_epoch, &md->rb_kernels, true));
            TGAP_CUDA(ctx, cudaGraphLaunch(md->exec_rb, ctx->stream));
            ctx->launches += md->rb_kernels;
            md->sys->nb.count_on_device = true;
        } else if (graphs) {
            CHECK_RC(md_graph(md, 1, &md->graph, &md->exec, &md->graph_epoch, &md->graph_kernels));
            TGAP_CUDA(ctx, cudaGraphLaunch(md->exec, ctx->stream));
            ctx->launches += md->graph_kernels;
        } else {
            CHECK_RC(md_step_body(md, rebuild && md->device_rebuild));
            md->settled_epoch = g_alloc_epoch.load(std::memory_order_relaxed);
        }
        ++md->step;
    }
    return TGAP_OK;
}

extern "C" int tgap_md_get_state(tgap_md *md, double *positions, double *velocities, double *forces,
                                 double *e_pot, double *e_kin)
{
    if (!md) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = md->ctx;
    CHECK_RC(activate(ctx));
    const int N = md->sys->nb.n_atoms;
    std::vector<double> v(3 * N), e(N), m(N);
    if (positions) CHECK_RC(download(ctx, positions, md->sys->nb.positions, 3 * (size_t)N));
    CHECK_RC(download(ctx, v.data(), md->vel, 3 * (size_t)N));
    if (forces) CHECK_RC(download(ctx, forces, md->forces, 3 * (size_t)N));
    CHECK_RC(download(ctx, e.data(), md->energies, (size_t)N));
    CHECK_RC(download(ctx, m.data(), md->mass, (size_t)N));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    CHECK_RC(read_device_check(ctx));
    if (velocities) std::memcpy(velocities, v.data(), sizeof(double) * 3 * N);
    double ep = 0.0, ek = 0.0;
    for (int i = 0; i < N; ++i) {
        ep += e[i];
        ek += 0.5 * m[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    }
    if (e_pot) *e_pot = ep;
    if (e_kin) *e_kin = ek;
    return TGAP_OK;
}

// ============================================================================ Monte Carlo

struct tgap_mc {
    tgap_context *ctx;
    tgap_system *sys;
    std::vector<tgap_model *> models;
    int precision, use_graph;
    double temperature, rc_sel, skin;
    int cap = 0, pmax = 0;
    int batch = 8, sized_batch = 0;  // speculative batch slots (plain GAP MC); slots the buffers hold
    int64_t rebuilds = 0;
    McModelSel sel{};
    DevBuf st, ecache, dacc, mark, sites, tstart, txyz, trjs, tnsp, etrial;
    std::vector<DevBuf> c, q, norm, q_hi, q_lo;  // per model, the trial rows
    std::vector<GapWork> gw;
    DevBuf patom, pdisp, pu, log_de, log_acc, log_des, log_stage;
    HostBuf hst;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t graph_epoch = 0;
    int64_t graph_kernels = 0;
    // learned screen (delayed acceptance); screened: installed (proposals carry deviate pairs),
    // screen_active: used by the step (off after a fallback to plain GAP MC)
    bool screened = false, screen_active = false;
    int64_t fb_window = 256;                      // screened proposals per fallback check
    double fb_min_confirm = 0.1, fb_min_pass = 0.002, fb_max_pass = 0.99;
    long long fb_prop0 = 0, fb_pass0 = 0, fb_conf0 = 0;  // counters at the start of the window
    int64_t fallbacks = 0;
    ScreenDev sd{};
    DevBuf s_mean, s_pca, s_w1, s_b1, s_w2, s_b2, s_w3, es_cache, es_trial;
    DevBuf tskip;  // per row tile of the trial rows: skipped by the exact GAP kernel (screened batch)
    int64_t last_n = 0;
};

constexpr int kMcBatch = 32;       // proposals per graph launch, one at a time (screened)
constexpr int kMcBatchSteps = 12;  // speculative batches per graph launch (plain GAP MC)

// Trial buffers for the current lists: pmax = longest list, cap = most sites one move can touch.
static int mc_size_trial(tgap_mc *mc)
{
    tgap_context *ctx = mc->ctx;
    NeighborBatch &nb = mc->sys->nb;
    const int N = nb.n_atoms;
    std::vector<int> nn(N);
    CHECK_RC(download(ctx, nn.data(), nb.n_neigh, (size_t)N));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int pmax = 1;
    for (int v : nn) pmax = std::max(pmax, v);
    if (pmax <= mc->pmax && mc->cap > 0 && mc->batch <= mc->sized_batch) return TGAP_OK;
    if (pmax > mc->pmax || mc->cap == 0) {
        mc->pmax = (pmax + 7) / 8 * 8 + 8;  // room for a few more pairs before resizing
        mc->cap = (mc->pmax + 1 + 31) / 32 * 32;
    }
    mc->sized_batch = std::max(mc->batch, 1);
    const int M = (int)mc->models.size(), cap = mc->cap, pm = mc->pmax;
    const int rows = mc->sized_batch * cap;  // trial rows per model: slots x cap
    const int rows_pad = (rows + 127) / 128 * 128;
    std::vector<int64_t> ts(rows + 1);
    for (int r = 0; r <= rows; ++r) ts[r] = (int64_t)r * pm;
    const size_t slots = (size_t)M * rows * pm;
    if (mc->sites.ensure(sizeof(int) * (size_t)M * rows) || mc->tstart.ensure(sizeof(int64_t) * (rows + 1)) ||
        mc->txyz.ensure(sizeof(double) * 3 * slots) || mc->trjs.ensure(sizeof(double) * slots) ||
        mc->tnsp.ensure(sizeof(int) * slots) || mc->etrial.ensure(sizeof(double) * (size_t)M * rows) ||
        mc->es_trial.ensure(sizeof(float) * (size_t)rows) ||
        mc->tskip.ensure(sizeof(int) * (size_t)((rows + 127) / 128)))
        return set_error(ctx, TGAP_ERR_NOMEM, "Monte Carlo trial buffers");
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->tnsp.ptr, 0, sizeof(int) * slots, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->trjs.ptr, 0, sizeof(double) * slots, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->txyz.ptr, 0, sizeof(double) * 3 * slots, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->sites.ptr, 0, sizeof(int) * (size_t)M * rows, ctx->stream));
    CHECK_RC(upload(ctx, mc->tstart, ts.data(), ts.size()));
    for (int m = 0; m < M; ++m) {
        const tgap_model *md = mc->models[m];
        const SoapParams &P = md->soap.p;
        const size_t nlm = (size_t)(P.l_max + 1) * (P.l_max + 1);
        const size_t tsz = mc->precision == TGAP_FP64 ? 8 : 4;
        const int q_ld = mc->precision == TGAP_FP64 ? md->gap.dim : md->gap.dim_pad;
        if (mc->c[m].ensure(tsz * rows * P.n_max * nlm) || mc->q[m].ensure(tsz * (size_t)rows_pad * q_ld) ||
            mc->norm[m].ensure(tsz * rows))
            return set_error(ctx, TGAP_ERR_NOMEM, "Monte Carlo trial buffers");
        if (mc->precision != TGAP_FP64) {
            if (mc->q_hi[m].ensure(2 * (size_t)rows_pad * q_ld) || mc->q_lo[m].ensure(2 * (size_t)rows_pad * q_ld))
                return set_error(ctx, TGAP_ERR_NOMEM, "Monte Carlo trial buffers");
            // rows past cap feed the 128-row GEMM tile: zero
            TGAP_CUDA(ctx, cudaMemsetAsync(mc->q_hi[m].ptr, 0, mc->q_hi[m].bytes, ctx->stream));
            TGAP_CUDA(ctx, cudaMemsetAsync(mc->q_lo[m].ptr, 0, mc->q_lo[m].bytes, ctx->stream));
        }
    }
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}

static McLogs mc_logs(tgap_mc *mc)
{
    return McLogs{mc->log_de.as<double>(), mc->log_acc.as<unsigned char>(), mc->log_des.as<double>(),
                  mc->log_stage.as<unsigned char>()};
}

// One proposal: select, trial geometry, descriptor rows and GAP energies per model (with the
// screen stage before the exact one when a screen is set), acceptance.
static int mc_step_body(tgap_mc *mc)
{
    tgap_context *ctx = mc->ctx;
    NeighborBatch &nb = mc->sys->nb;
    const int M = (int)mc->models.size(), cap = mc->cap, pm = mc->pmax, N = nb.n_atoms;
    McDev *st = mc->st.as<McDev>();
    CHECK_RC(mc_select(ctx, st, nb, mc->sel, mc->rc_sel, mc->skin, mc->patom.as<int>(), mc->pdisp.as<double>(),
                       mc->dacc.as<double>(), mc->mark.as<long long>(), mc->sites.as<int>(), cap));
    CHECK_RC(mc_trial_geometry(ctx, st, nb, M, mc->sites.as<int>(), cap, pm, mc->txyz.as<double>(),
                               mc->trjs.as<double>(), mc->tnsp.as<int>()));
    for (int m = 0; m < M; ++m) {
        const tgap_model *md = mc->models[m];
        const size_t off = (size_t)m * cap * pm;
        PairView pv{mc->tstart.as<int64_t>(), mc->txyz.as<double>() + 3 * off, mc->trjs.as<double>() + off,
                    mc->tnsp.as<int>() + off, nullptr, 0, ctx->d_check};
        SoapOut o;
        o.c = mc->c[m].ptr;
        o.q = mc->q[m].ptr;
        o.norm = mc->norm[m].ptr;
        double *e_rows = mc->etrial.as<double>() + (size_t)m * cap;
        if (mc->precision == TGAP_FP64) {
            o.q_ld = md->gap.dim;
            CHECK_RC(soap_forward(ctx, md->soap, pv, nullptr, cap, TGAP_FP64, o));
            CHECK_RC(gap_energy_grad_f64(ctx, md->gap, (const double *)o.q, o.q_ld, cap, 0.0, 0, &mc->gw[m], nullptr,
                                         e_rows, nullptr));
        } else {
            o.q_ld = md->gap.dim_pad;
            o.q_hi = mc->q_hi[m].as<__nv_bfloat16>();
            o.q_lo = mc->q_lo[m].as<__nv_bfloat16>();
            CHECK_RC(soap_forward(ctx, md->soap, pv, nullptr, cap, TGAP_MIXED, o));
            const int *skip = nullptr;
            if (mc->screen_active) {
                // stage 1 on the trial rows' screen energies; a rejection skips the exact GEMM
                const int *d_count = reinterpret_cast<const int *>(reinterpret_cast<const char *>(st) +
                                                                   offsetof(McDev, count));
                CHECK_RC(screen_rows(ctx, mc->sd, (const float *)o.q, o.q_ld, cap, d_count, mc->es_trial.as<float>()));
                CHECK_RC(mc_screen_stage(ctx, st, mc->sites.as<int>(), mc->es_trial.as<float>(),
                                         mc->es_cache.as<float>(), mc->pu.as<double>(), mc->temperature, mc_logs(mc)));
                skip = reinterpret_cast<const int *>(reinterpret_cast<const char *>(st) + offsetof(McDev, skip));
            }
            CHECK_RC(gap_energy_grad_mixed(ctx, md->gap, o.q_hi, o.q_lo, cap, 0.0, 0, &mc->gw[m], nullptr, e_rows,
                                           nullptr, skip));
        }
    }
    return mc_accept(ctx, st, M, mc->sites.as<int>(), cap, mc->etrial.as<double>(), mc->ecache.as<double>(), N,
                     nb.positions.as<double>(), mc->dacc.as<double>(), mc->pu.as<double>(), mc->temperature,
                     mc_logs(mc), mc->screen_active ? 1 : 0, mc->screened ? 2 : 1, mc->es_trial.as<float>(),
                     mc->es_cache.as<float>());
}

// One speculative batch of plain GAP MC (mc_select_batch): select, trial geometry, descriptor rows
// and GAP energies of every slot per model, then the in-order settlement.
static int mc_step_body_batch(tgap_mc *mc)
{
    tgap_context *ctx = mc->ctx;
    NeighborBatch &nb = mc->sys->nb;
    const int M = (int)mc->models.size(), cap = mc->cap, pm = mc->pmax, B = mc->batch, rows = B * cap;
    McDev *st = mc->st.as<McDev>();
    CHECK_RC(mc_select_batch(ctx, st, nb, mc->sel, mc->rc_sel, mc->skin, mc->patom.as<int>(), mc->pdisp.as<double>(),
                             mc->dacc.as<double>(), mc->mark.as<long long>(), mc->sites.as<int>(), cap, B));
    CHECK_RC(mc_trial_geometry_batch(ctx, st, nb, M, mc->sites.as<int>(), cap, pm, B, mc->txyz.as<double>(),
                                     mc->trjs.as<double>(), mc->tnsp.as<int>()));
    for (int m = 0; m < M; ++m) {
        const tgap_model *md = mc->models[m];
        const size_t off = (size_t)m * rows * pm;
        PairView pv{mc->tstart.as<int64_t>(), mc->txyz.as<double>() + 3 * off, mc->trjs.as<double>() + off,
                    mc->tnsp.as<int>() + off, nullptr, 0, ctx->d_check};
        SoapOut o;
        o.c = mc->c[m].ptr;
        o.q = mc->q[m].ptr;
        o.norm = mc->norm[m].ptr;
        double *e_rows = mc->etrial.as<double>() + (size_t)m * rows;
        if (mc->precision == TGAP_FP64) {
            o.q_ld = md->gap.dim;
            CHECK_RC(soap_forward(ctx, md->soap, pv, nullptr, rows, TGAP_FP64, o));
            CHECK_RC(gap_energy_grad_f64(ctx, md->gap, (const double *)o.q, o.q_ld, rows, 0.0, 0, &mc->gw[m], nullptr,
                                         e_rows, nullptr));
        } else {
            o.q_ld = md->gap.dim_pad;
            o.q_hi = mc->q_hi[m].as<__nv_bfloat16>();
            o.q_lo = mc->q_lo[m].as<__nv_bfloat16>();
            CHECK_RC(soap_forward(ctx, md->soap, pv, nullptr, rows, TGAP_MIXED, o));
            const int *skip_tiles = nullptr;
            if (mc->screen_active) {
                // delayed acceptance, stage 1 of every slot from the screen energies of its rows;
                // the exact GAP kernel skips the row tiles of slots the screen rejects
                const int n_tiles = (rows + 127) / 128;
                CHECK_RC(screen_rows(ctx, mc->sd, (const float *)o.q, o.q_ld, rows, nullptr, mc->es_trial.as<float>()));
                CHECK_RC(mc_screen_batch(ctx, st, mc->sites.as<int>(), cap, B, mc->es_trial.as<float>(),
                                         mc->es_cache.as<float>(), mc->pu.as<double>(), mc->temperature,
                                         mc->tskip.as<int>(), n_tiles));
                skip_tiles = mc->tskip.as<int>();
            }
            CHECK_RC(gap_energy_grad_mixed(ctx, md->gap, o.q_hi, o.q_lo, rows, 0.0, 0, &mc->gw[m], nullptr, e_rows,
                                           nullptr, nullptr, false, skip_tiles));
        }
    }
    return mc_resolve_batch(ctx, st, nb, M, mc->sites.as<int>(), cap, B, mc->etrial.as<double>(),
                            mc->ecache.as<double>(), nb.positions.as<double>(), mc->dacc.as<double>(),
                            mc->pu.as<double>(), mc->screened ? 2 : 1, mc->temperature, mc->rc_sel, mc->skin,
                            mc_logs(mc), mc->screen_active ? 1 : 0, mc->es_trial.as<float>(),
                            mc->es_cache.as<float>());
}

static void mc_drop_graph(tgap_mc *mc)
{
    if (mc->exec) cudaGraphExecDestroy(mc->exec);
    if (mc->graph) cudaGraphDestroy(mc->graph);
    mc->exec = nullptr;
    mc->graph = nullptr;
}

// Fallback to plain GAP MC when the screen's acceptance collapses, or when it settles almost
// nothing: over each window of fb_window screened proposals, the fraction passed to the exact stage
// (pass) and the fraction of those the exact energies confirm (confirm). Either falling below its
// floor switches the screen off, and so does pass above fb_max_pass (delayed acceptance saves only
// the exact evaluations of the proposals the screen rejects; when it rejects fewer than 1 - max_pass
// of them, its own evaluation costs more than it saves). The chain's target distribution is the
// same either way, so the switch may happen at any proposal boundary. Returns true when it switched.
static bool mc_screen_check(tgap_mc *mc, const McDev &h)
{
    if (!mc->screen_active) return false;
    const long long np = h.s_prop - mc->fb_prop0;
    if (np < mc->fb_window) return false;
    const long long npass = h.s_pass - mc->fb_pass0, nconf = h.s_conf - mc->fb_conf0;
    const double pass = (double)npass / (double)np;
    const double confirm = npass > 0 ? (double)nconf / (double)npass : 1.0;
    mc->fb_prop0 = h.s_prop;
    mc->fb_pass0 = h.s_pass;
    mc->fb_conf0 = h.s_conf;
    if (pass >= mc->fb_min_pass && pass <= mc->fb_max_pass && (npass < 32 || confirm >= mc->fb_min_confirm))
        return false;
    mc->screen_active = false;
    ++mc->fallbacks;
    mc_drop_graph(mc);
    return true;
}

static int mc_read_state(tgap_mc *mc, McDev *out)
{
    tgap_context *ctx = mc->ctx;
    TGAP_CUDA(ctx, cudaMemcpyAsync(mc->hst.ptr, mc->st.ptr, sizeof(McDev), cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(out, mc->hst.ptr, sizeof(McDev));
    return read_device_check(ctx);
}

extern "C" int tgap_mc_create(tgap_context *ctx, tgap_system *sys, int n_models, tgap_model *const *models,
                              double temperature, int precision, int use_graph, tgap_mc **out)
{
    CHECK_RC(activate(ctx));
    if (!sys || n_models <= 0 || n_models > kMcMaxModels || !models || !(temperature > 0) || !out)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_mc_create: bad arguments");
    if (precision != TGAP_FP64 && precision != TGAP_MIXED)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_mc_create: precision");
    if (!sys->nb.replicated)
        return set_error(ctx, TGAP_ERR_UNSUPPORTED, "Monte Carlo needs a system built from primitive cells");
    if (sys->range_beg != 0 || sys->range_end >= 0)
        return set_error(ctx, TGAP_ERR_UNSUPPORTED, "Monte Carlo needs every site (tgap_system_set_site_range)");
    double rc = 0.0;
    for (int m = 0; m < n_models; ++m) rc = std::max(rc, models[m]->soap.p.rcut_max);
    if (!(sys->rcut > rc))
        return set_error(ctx, TGAP_ERR_ARGUMENT, "Monte Carlo needs a neighbor skin: system cutoff %g <= model %g",
                         sys->rcut, rc);
    auto *mc = new tgap_mc();
    std::unique_ptr<tgap_mc, int (*)(tgap_mc *)> guard(mc, tgap_mc_destroy);
    mc->ctx = ctx;
    mc->sys = sys;
    mc->models.assign(models, models + n_models);
    mc->precision = precision;
    mc->use_graph = use_graph;
    mc->temperature = temperature;
    mc->rc_sel = rc;
    mc->skin = sys->rcut - rc;
    mc->sel.n_models = n_models;
    // speculative batch width: the FP32/bf16 rows are cheap enough that 12 side-by-side
    // proposals cost little more than one; FP64 rows are not (measured on the 1000-atom MC box)
    mc->batch = precision == TGAP_MIXED ? 12 : 4;
    for (int m = 0; m < n_models; ++m) {
        mc->sel.central_species[m] = models[m]->central_species;
        if (precision == TGAP_MIXED && !models[m]->mixed_ready)
            return set_error(ctx, TGAP_ERR_UNSUPPORTED, "mixed path not prepared");
    }
    mc->c.resize(n_models);
    mc->q.resize(n_models);
    mc->norm.resize(n_models);
    mc->q_hi.resize(n_models);
    mc->q_lo.resize(n_models);
    mc->gw.resize(n_models);
    const int N = sys->nb.n_atoms;
    if (mc->st.ensure(sizeof(McDev)) || mc->ecache.ensure(sizeof(double) * (size_t)n_models * N) ||
        mc->dacc.ensure(sizeof(double) * N) || mc->mark.ensure(sizeof(long long) * (size_t)kMcMaxBatch * N) ||
        mc->hst.ensure(sizeof(McDev)))
        return set_error(ctx, TGAP_ERR_NOMEM, "Monte Carlo state");
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->st.ptr, 0, sizeof(McDev), ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->ecache.ptr, 0, sizeof(double) * (size_t)n_models * N, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->dacc.ptr, 0, sizeof(double) * N, ctx->stream));
    TGAP_CUDA(ctx, cudaMemsetAsync(mc->mark.ptr, 0, sizeof(long long) * (size_t)kMcMaxBatch * N, ctx->stream));
    // fresh lists at the current positions, then the cached site energies of every model
    CHECK_RC(tgap_system_update(sys, 1));
    for (int m = 0; m < n_models; ++m)
        CHECK_RC(compute_model(ctx, sys, models[m], precision, 0, mc->ecache.as<double>() + (size_t)m * N, nullptr,
                               nullptr));
    CHECK_RC(mc_size_trial(mc));
    *out = guard.release();
    return TGAP_OK;
}

extern "C" int tgap_mc_destroy(tgap_mc *mc)
{
    if (!mc) return TGAP_OK;
    cudaSetDevice(mc->ctx->device);
    cudaStreamSynchronize(mc->ctx->stream);
    if (mc->exec) cudaGraphExecDestroy(mc->exec);
    if (mc->graph) cudaGraphDestroy(mc->graph);
    DevBuf *bufs[] = {&mc->st, &mc->ecache, &mc->dacc, &mc->mark, &mc->sites, &mc->tstart, &mc->txyz, &mc->trjs,
                      &mc->tnsp, &mc->etrial, &mc->patom, &mc->pdisp, &mc->pu, &mc->log_de, &mc->log_acc,
                      &mc->log_des, &mc->log_stage, &mc->s_mean, &mc->s_pca, &mc->s_w1, &mc->s_b1, &mc->s_w2,
                      &mc->s_b2, &mc->s_w3, &mc->es_cache, &mc->es_trial, &mc->tskip};
    for (DevBuf *b : bufs) b->release();
    for (auto *v : {&mc->c, &mc->q, &mc->norm, &mc->q_hi, &mc->q_lo})
        for (DevBuf &b : *v) b.release();
    for (GapWork &w : mc->gw) {
        DevBuf *wb[] = {&w.e_part, &w.G, &w.g, &w.G_hi, &w.G_lo};
        for (DevBuf *b : wb) b->release();
    }
    mc->hst.release();
    delete mc;
    return TGAP_OK;
}

extern "C" int tgap_mc_run(tgap_mc *mc, int64_t n, const int *atoms, const double *disp, const double *uniform,
                           int64_t *n_accepted, double *de_log, unsigned char *acc_log)
{
    if (!mc || n < 0 || (n > 0 && (!atoms || !disp || !uniform))) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = mc->ctx;
    CHECK_RC(activate(ctx));
    if (n == 0) {
        if (n_accepted) *n_accepted = 0;
        return TGAP_OK;
    }
    const int N = mc->sys->nb.n_atoms;
    for (int64_t k = 0; k < n; ++k) {
        if (atoms[k] < 0 || atoms[k] >= N) return set_error(ctx, TGAP_ERR_ARGUMENT, "proposal %lld: atom", (long long)k);
        // a move of |d| >= skin could bring a pair into the cutoff that no skin-padded list holds,
        // even right after a rebuild
        const double d2 = disp[3 * k] * disp[3 * k] + disp[3 * k + 1] * disp[3 * k + 1] + disp[3 * k + 2] * disp[3 * k + 2];
        if (!(d2 < mc->skin * mc->skin))
            return set_error(ctx, TGAP_ERR_ARGUMENT,
                             "proposal %lld: displacement %g A is not below the neighbor skin %g A (system cutoff "
                             "minus model cutoff)",
                             (long long)k, std::sqrt(d2), mc->skin);
    }
    const size_t nu = (mc->screened ? 2 : 1) * (size_t)n;  // two deviates per proposal with a screen
    if (mc->patom.ensure(sizeof(int) * n) || mc->pdisp.ensure(sizeof(double) * 3 * n) ||
        mc->pu.ensure(sizeof(double) * nu) || mc->log_de.ensure(sizeof(double) * n) || mc->log_acc.ensure(n) ||
        mc->log_des.ensure(sizeof(double) * n) || mc->log_stage.ensure(n))
        return set_error(ctx, TGAP_ERR_NOMEM, "Monte Carlo proposals");
    CHECK_RC(upload(ctx, mc->patom, atoms, (size_t)n));
    CHECK_RC(upload(ctx, mc->pdisp, disp, 3 * (size_t)n));
    CHECK_RC(upload(ctx, mc->pu, uniform, nu));
    mc->last_n = n;
    McDev h;
    CHECK_RC(mc_read_state(mc, &h));
    const long long acc0 = h.accepted;
    CHECK_RC(mc_begin(ctx, mc->st.as<McDev>(), n));
    long long rebuilt_at = -1;  // proposals settled at the last rebuild
    for (;;) {
        CHECK_RC(mc_read_state(mc, &h));
        // every proposal below next is settled except the deferred ones
        const long long settled_now = h.next - h.n_pend;
        if (h.status == kMcNeedRebuild) {
            // fresh lists always admit the first unsettled move (below the skin); a second request
            // with nothing settled in between means the state is inconsistent, not that another
            // rebuild would help
            if (rebuilt_at == settled_now)
                return set_error(ctx, TGAP_ERR_NUMERIC, "proposal %lld still needs a list rebuild after one",
                                 h.n_pend > 0 ? h.pend[0] : h.next);
            rebuilt_at = settled_now;
            // lists at the current positions; the cached site energies stay valid
            NeighborBatch &nb = mc->sys->nb;
            CHECK_RC(neighbors_sync_positions(ctx, &nb));
            int64_t n_pairs = 0;
            CHECK_RC(neighbors_rebuild_lists(ctx, &nb, -1, &n_pairs));
            CHECK_RC(neighbors_geometry(ctx, &nb, false, false));
            CHECK_RC(mc_lists_rebuilt(ctx, mc->st.as<McDev>(), mc->dacc.as<double>(), N));
            CHECK_RC(mc_size_trial(mc));
            ++mc->rebuilds;
            continue;
        }
        if (h.status == kMcDone || (h.next >= n && h.n_pend == 0)) break;
        mc_screen_check(mc, h);
        if (mc->use_graph) {
            if (!mc->exec || mc->graph_epoch != g_alloc_epoch.load(std::memory_order_relaxed)) {
                if (mc->exec) cudaGraphExecDestroy(mc->exec);
                if (mc->graph) cudaGraphDestroy(mc->graph);
                mc->exec = nullptr;
                mc->graph = nullptr;
                const uint64_t epoch = g_alloc_epoch.load(std::memory_order_relaxed);
                TGAP_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
                const int64_t launches = ctx->launches;
                int rc = TGAP_OK;
                if (mc->screen_active && mc->batch <= 1)
                    for (int b = 0; b < kMcBatch && !rc; ++b) rc = mc_step_body(mc);
                else
                    for (int b = 0; b < kMcBatchSteps && !rc; ++b) rc = mc_step_body_batch(mc);
                cudaGraph_t g = nullptr;
                cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
                mc->graph_kernels = ctx->launches - launches;
                ctx->launches = launches;
                if (rc) {
                    if (g) cudaGraphDestroy(g);
                    return rc;
                }
                if (ce != cudaSuccess) return cuda_check(ctx, ce, "graph capture");
                // a buffer allocated during the capture would not be in the graph's view
                if (g_alloc_epoch.load(std::memory_order_relaxed) != epoch) {
                    cudaGraphDestroy(g);
                    continue;
                }
                mc->graph = g;
                TGAP_CUDA(ctx, cudaGraphInstantiate(&mc->exec, g, 0));
                mc->graph_epoch = epoch;
            }
            TGAP_CUDA(ctx, cudaGraphLaunch(mc->exec, ctx->stream));
            ctx->launches += mc->graph_kernels;
        } else if (mc->screen_active && mc->batch <= 1) {
            for (int b = 0; b < kMcBatch; ++b) CHECK_RC(mc_step_body(mc));
        } else {
            for (int b = 0; b < kMcBatchSteps; ++b) CHECK_RC(mc_step_body_batch(mc));
        }
    }
    if (de_log) CHECK_RC(download(ctx, de_log, mc->log_de, (size_t)n));
    if (acc_log) TGAP_CUDA(ctx, cudaMemcpyAsync(acc_log, mc->log_acc.ptr, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (n_accepted) *n_accepted = h.accepted - acc0;
    return read_device_check(ctx);
}

extern "C" int tgap_mc_get_state(tgap_mc *mc, double *positions, double *energies, double *e_total,
                                 int64_t *accepted, int64_t *rebuilds)
{
    if (!mc) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = mc->ctx;
    CHECK_RC(activate(ctx));
    const int N = mc->sys->nb.n_atoms, M = (int)mc->models.size();
    std::vector<double> e((size_t)M * N);
    if (positions) CHECK_RC(download(ctx, positions, mc->sys->nb.positions, 3 * (size_t)N));
    CHECK_RC(download(ctx, e.data(), mc->ecache, e.size()));
    McDev h;
    CHECK_RC(mc_read_state(mc, &h));
    double tot = 0.0;
    const std::vector<double> &e0 = mc->sys->host_e0;  // calculate_e0: constant under moves
    for (int i = 0; i < N; ++i) {
        double v = 0.0;
        for (int m = 0; m < M; ++m) v += e[(size_t)m * N + i];
        if (!e0.empty()) v += e0[i];
        if (energies) energies[i] = v;
        tot += v;
    }
    if (e_total) *e_total = tot;
    if (accepted) *accepted = h.accepted;
    if (rebuilds) *rebuilds = mc->rebuilds;
    return TGAP_OK;
}

extern "C" int tgap_mc_set_screen(tgap_mc *mc, int dim, int n_pca, int n_hidden, const float *mean, const float *pca,
                                  const float *w1, const float *b1, const float *w2, const float *b2,
                                  const float *w3, float b3)
{
    if (!mc) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = mc->ctx;
    CHECK_RC(activate(ctx));
    if (!mean || !pca || !w1 || !b1 || !w2 || !b2 || !w3 || n_pca < 1 || n_pca > kScreenMaxPca || n_hidden < 1 ||
        n_hidden > kScreenMaxHidden)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "tgap_mc_set_screen: bad arguments");
    if (mc->precision != TGAP_MIXED || mc->models.size() != 1 || mc->models[0]->central_species != 0 ||
        mc->models[0]->gap.dim_pad > 384)
        return set_error(ctx, TGAP_ERR_UNSUPPORTED,
                         "the screen needs the mixed path, one model over all sites and a descriptor of <= 384");
    const tgap_model *md = mc->models[0];
    if (dim != md->gap.dim) return set_error(ctx, TGAP_ERR_ARGUMENT, "screen dim %d != descriptor %d", dim, md->gap.dim);
    if (screen_smem_bytes(dim, n_pca, n_hidden) > 227 * 1024)
        return set_error(ctx, TGAP_ERR_ARGUMENT, "screen too large for one CTA's shared memory");
    // bf16, transposed to input-index-major (the kernel reads along the output index)
    auto to_bf16_t = [](const float *x, size_t rows, size_t cols) {
        std::vector<__nv_bfloat16> v(rows * cols);
        for (size_t r = 0; r < rows; ++r)
            for (size_t c = 0; c < cols; ++c) v[c * rows + r] = __float2bfloat16_rn(x[r * cols + c]);
        return v;
    };
    const auto vp = to_bf16_t(pca, n_pca, dim), v1 = to_bf16_t(w1, n_hidden, n_pca),
               v2 = to_bf16_t(w2, n_hidden, n_hidden), v3 = to_bf16_t(w3, n_hidden, 1);
    CHECK_RC(upload(ctx, mc->s_mean, mean, (size_t)dim));
    CHECK_RC(upload(ctx, mc->s_pca, vp.data(), vp.size()));
    CHECK_RC(upload(ctx, mc->s_w1, v1.data(), v1.size()));
    CHECK_RC(upload(ctx, mc->s_b1, b1, (size_t)n_hidden));
    CHECK_RC(upload(ctx, mc->s_w2, v2.data(), v2.size()));
    CHECK_RC(upload(ctx, mc->s_b2, b2, (size_t)n_hidden));
    CHECK_RC(upload(ctx, mc->s_w3, v3.data(), v3.size()));
    mc->sd = ScreenDev{dim, n_pca, n_hidden, mc->s_mean.as<float>(), mc->s_pca.as<__nv_bfloat16>(),
                       mc->s_w1.as<__nv_bfloat16>(), mc->s_b1.as<float>(), mc->s_w2.as<__nv_bfloat16>(),
                       mc->s_b2.as<float>(), mc->s_w3.as<__nv_bfloat16>(), b3};
    // screen energies of every atom at the current positions (FP32 descriptors of the mixed path)
    tgap_system *sys = mc->sys;
    const int N = sys->nb.n_atoms;
    if (mc->es_cache.ensure(sizeof(float) * N) ||
        mc->es_trial.ensure(sizeof(float) * (size_t)std::max(mc->sized_batch, 1) * mc->cap))
        return set_error(ctx, TGAP_ERR_NOMEM, "screen caches");
    CHECK_RC(neighbors_refresh(ctx, &sys->nb));
    DevBuf c, q, norm;
    std::unique_ptr<DevBuf, void (*)(DevBuf *)> gc(&c, [](DevBuf *b) { b->release(); });
    std::unique_ptr<DevBuf, void (*)(DevBuf *)> gq(&q, [](DevBuf *b) { b->release(); });
    std::unique_ptr<DevBuf, void (*)(DevBuf *)> gn(&norm, [](DevBuf *b) { b->release(); });
    const SoapParams &P = md->soap.p;
    const size_t nlm = (size_t)(P.l_max + 1) * (P.l_max + 1);
    if (c.ensure(4 * (size_t)N * P.n_max * nlm) || q.ensure(4 * (size_t)N * md->gap.dim_pad) || norm.ensure(4 * (size_t)N))
        return set_error(ctx, TGAP_ERR_NOMEM, "screen initialisation");
    PairView pv{sys->nb.start.as<int64_t>(), sys->nb.xyz.as<double>(), sys->nb.rjs.as<double>(),
                sys->nb.nspecies.as<int>(), sys->nb.jatom.as<int>(), N, ctx->d_check};
    SoapOut o;
    o.c = c.ptr;
    o.q = q.ptr;
    o.norm = norm.ptr;
    o.q_ld = md->gap.dim_pad;
    CHECK_RC(soap_forward(ctx, md->soap, pv, nullptr, N, TGAP_MIXED, o));
    CHECK_RC(screen_rows(ctx, mc->sd, q.as<float>(), o.q_ld, N, nullptr, mc->es_cache.as<float>()));
    McDev h;
    CHECK_RC(mc_read_state(mc, &h));
    mc->screened = true;
    mc->screen_active = true;
    mc->fb_prop0 = h.s_prop;
    mc->fb_pass0 = h.s_pass;
    mc->fb_conf0 = h.s_conf;
    mc_drop_graph(mc);  // the per-proposal graph changes shape
    return TGAP_OK;
}

extern "C" int tgap_mc_screen_fallback(tgap_mc *mc, int64_t window, double min_confirm, double min_pass,
                                       double max_pass)
{
    if (!mc || window < 1 || !(min_confirm >= 0.0 && min_confirm <= 1.0) || !(min_pass >= 0.0 && min_pass <= 1.0) ||
        !(max_pass >= min_pass && max_pass <= 1.0))
        return TGAP_ERR_ARGUMENT;
    mc->fb_window = window;
    mc->fb_min_confirm = min_confirm;
    mc->fb_min_pass = min_pass;
    mc->fb_max_pass = max_pass;
    return TGAP_OK;
}

extern "C" int tgap_mc_set_batch(tgap_mc *mc, int slots)
{
    if (!mc || slots < 1 || slots > kMcMaxBatch) return TGAP_ERR_ARGUMENT;
    CHECK_RC(activate(mc->ctx));
    mc->batch = slots;
    CHECK_RC(mc_size_trial(mc));
    mc_drop_graph(mc);
    return TGAP_OK;
}

extern "C" int tgap_mc_batch_stats(tgap_mc *mc, int64_t *batches, int64_t *settled)
{
    if (!mc) return TGAP_ERR_ARGUMENT;
    CHECK_RC(activate(mc->ctx));
    McDev h;
    CHECK_RC(mc_read_state(mc, &h));
    if (batches) *batches = h.batches;
    if (settled) *settled = h.batch_resolved;
    return TGAP_OK;
}

extern "C" int tgap_mc_screen_stats(tgap_mc *mc, int *active, int64_t *judged, int64_t *passed, int64_t *confirmed,
                                    int64_t *fallbacks)
{
    if (!mc) return TGAP_ERR_ARGUMENT;
    CHECK_RC(activate(mc->ctx));
    McDev h;
    CHECK_RC(mc_read_state(mc, &h));
    if (active) *active = mc->screen_active ? 1 : 0;
    if (judged) *judged = h.s_prop;
    if (passed) *passed = h.s_pass;
    if (confirmed) *confirmed = h.s_conf;
    if (fallbacks) *fallbacks = mc->fallbacks;
    return TGAP_OK;
}

extern "C" int tgap_mc_screen_log(tgap_mc *mc, int64_t n, double *de_screen, unsigned char *stage)
{
    if (!mc || n < 0 || n > mc->last_n) return TGAP_ERR_ARGUMENT;
    tgap_context *ctx = mc->ctx;
    CHECK_RC(activate(ctx));
    if (de_screen) CHECK_RC(download(ctx, de_screen, mc->log_des, (size_t)n));
    if (stage) TGAP_CUDA(ctx, cudaMemcpyAsync(stage, mc->log_stage.ptr, (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    TGAP_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TGAP_OK;
}
