// C-ABI entry points of libspring_b200.so: context, inputs, orchestration.
// Kernels live in k_*.cu; this file validates arguments, owns device memory
// and sequences the launches on the context's stream.
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <new>

#include "spring_internal.cuh"

using namespace spring;

namespace spring {

HostConst host_constants() {
    HostConst k;
    const double pi = 4.0 * std::atan(1.0);
    k.wTHz = std::sqrt(1.60217733 * 6.02214076 * 10.0) * 10.0;
    k.vg_ms = k.wTHz * 100.0;
    k.BEConv = std::sqrt(1.60217733 * 6.02214076 * 10.0) * 6.582119569 * 100.0 / 8.617333262;
    k.Sctr3THz2 = 1.054571817 * (1.60217733 * 1.60217733) * (6.02214076 * 6.02214076 * 6.02214076) * 1000000.0 *
                  pi * 0.0625;
    const double hb = 1.054571817 * 1.602176565;
    const double na = 6.022140857;
    k.Sctr4THz2 = 0.125 * pi * (hb * hb) * (na * na * na * na) * 1000000.0;
    k.kW_m_k = (1.054571817 * 1.054571817) * 0.001 / 1.380649;
    return k;
}

int fail(spring_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int cuda_fail(spring_ctx* c, cudaError_t e, const char* what) {
    return fail(c, SPRING_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

static bool injected(spring_ctx* c, int kind) {
    if (c->inject_kind != kind || c->inject_n <= 0) return false;
    c->inject_seen[kind] += 1;
    if (c->inject_seen[kind] == c->inject_n) {
        c->inject_kind = -1;
        return true;
    }
    return false;
}

int dalloc_bytes(spring_ctx* c, void** p, size_t bytes, const char* what) {
    if (injected(c, 0)) return fail(c, SPRING_ERR_INJECTED, "%s: injected allocation failure", what);
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(c, SPRING_ERR_ALLOC, "%s: cudaMalloc(%zu bytes) failed: %s", what, bytes, cudaGetErrorString(e));
    }
    return SPRING_OK;
}

// Host -> device copy of `bytes` at `src`.  The bytes are first copied on the CPU into the context's
// pinned staging ring and the asynchronous copy reads them from there, so the caller's memory (and
// any temporary of the library) may be reused as soon as this returns, whatever kind of host memory
// it is, and the copy never waits for the stream.  Ring bytes are overwritten only once every copy
// queued from them has completed (ev_stage, recorded behind each staged copy).
int h2d(spring_ctx* c, void* dst, const void* src, size_t bytes, const char* what) {
    if (injected(c, 1)) return fail(c, SPRING_ERR_INJECTED, "%s: injected copy failure", what);
    if (bytes == 0) return SPRING_OK;
    if (!c->ev_stage) {
        cudaError_t e = cudaEventCreateWithFlags(&c->ev_stage, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(c, e, what);
    }
    const size_t need = (bytes + 255) & ~(size_t)255;
    if (c->h_stage_off + need > c->h_stage_cap) {
        // wrap (or grow): every copy queued from the ring must have read its bytes first
        if (c->stage_pending) {
            cudaError_t e = cudaEventSynchronize(c->ev_stage);
            if (e != cudaSuccess) return cuda_fail(c, e, what);
            c->stage_pending = false;
        }
        c->h_stage_off = 0;
        if (need > c->h_stage_cap) {
            if (c->h_stage) cudaFreeHost(c->h_stage);
            c->h_stage = nullptr;
            c->h_stage_cap = 0;
            const size_t cap = std::max<size_t>(need, (size_t)4 << 20);
            cudaError_t e = cudaHostAlloc((void**)&c->h_stage, cap, cudaHostAllocDefault);
            if (e != cudaSuccess) return cuda_fail(c, e, what);
            c->h_stage_cap = cap;
        }
    }
    char* st = c->h_stage + c->h_stage_off;
    std::memcpy(st, src, bytes);
    c->h_stage_off += need;
    cudaError_t e = cudaMemcpyAsync(dst, st, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_stage, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, what);
    c->stage_pending = true;
    return SPRING_OK;
}

int d2h(spring_ctx* c, void* dst, const void* src, size_t bytes, const char* what) {
    if (injected(c, 1)) return fail(c, SPRING_ERR_INJECTED, "%s: injected copy failure", what);
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, what);
}

__global__ void k_sum2(const int* __restrict__ a, const int* __restrict__ b, int* __restrict__ out) { *out = *a + *b; }

// *a + *b of two device ints with one readback.
int d2h_sum2(spring_ctx* c, const int* a, const int* b, int* out, const char* what) {
    SPRING_CHECK(dalloc(c, c->d_scr_sum, 1, what));
    k_sum2<<<1, 1, 0, c->stream>>>(a, b, c->d_scr_sum.p);
    SPRING_CHECK(launch_check(c, "k_sum2"));
    return d2h(c, out, c->d_scr_sum.p, sizeof(int), what);
}

int d2h_pin_async(spring_ctx* c, const void* src, size_t bytes, const char* what) {
    if (injected(c, 1)) return fail(c, SPRING_ERR_INJECTED, "%s: injected copy failure", what);
    const size_t n = (bytes + sizeof(int) - 1) / sizeof(int);
    if (c->h_pin_n < n) {
        if (c->h_pin) cudaFreeHost(c->h_pin);
        c->h_pin = nullptr;
        c->h_pin_n = 0;
        cudaError_t e = cudaHostAlloc((void**)&c->h_pin, std::max<size_t>(n, 1024) * sizeof(int), cudaHostAllocDefault);
        if (e != cudaSuccess) return cuda_fail(c, e, what);
        c->h_pin_n = std::max<size_t>(n, 1024);
    }
    if (!c->ev_aux) {
        cudaError_t e = cudaEventCreateWithFlags(&c->ev_aux, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(c, e, what);
    }
    cudaError_t e = cudaMemcpyAsync(c->h_pin, src, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_aux, c->stream);
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, what);
}

int pin_wait(spring_ctx* c, const char* what) {
    cudaError_t e = cudaEventSynchronize(c->ev_aux);
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, what);
}

int zero(spring_ctx* c, void* dst, size_t bytes, const char* what) {
    cudaError_t e = cudaMemsetAsync(dst, 0, bytes, c->stream);
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, what);
}

bool launch_injected(spring_ctx* c) {
    if (injected(c, 2)) return true;
    if (c->profiling && !c->prof_pending) {
        if (cudaEventCreate(&c->prof_pending) == cudaSuccess) cudaEventRecord(c->prof_pending, c->stream);
        else c->prof_pending = nullptr;
    }
    return false;
}

int launch_check(spring_ctx* c, const char* what) {
    c->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (c->profiling && c->prof_pending) {
        cudaEvent_t stop;
        if (cudaEventCreate(&stop) == cudaSuccess) {
            cudaEventRecord(stop, c->stream);
            c->prof.push_back({what, c->prof_pending, stop});
        } else {
            cudaEventDestroy(c->prof_pending);
        }
        c->prof_pending = nullptr;
    }
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, what);
}

void free_phonons(Phonons& p) {
    dfree(p.evec); dfree(p.omega); dfree(p.oneby); dfree(p.nbe); dfree(p.vel);
    p.set = false;
}

int alloc_phonons(spring_ctx* c, Phonons& p, int n) {
    p.n = n;
    const size_t nd = c->ndof;
    SPRING_CHECK(dalloc(c, p.evec, (size_t)n * nd * nd, "phonon eigenvectors"));
    SPRING_CHECK(dalloc(c, p.omega, (size_t)n * nd, "phonon omega"));
    SPRING_CHECK(dalloc(c, p.oneby, (size_t)n * nd, "phonon 1/omega"));
    SPRING_CHECK(dalloc(c, p.nbe, (size_t)c->nT * n * nd, "phonon nBE"));
    SPRING_CHECK(dalloc(c, p.vel, (size_t)n * nd * 3, "phonon velocity"));
    return SPRING_OK;
}

void clear_profile(spring_ctx* c) {
    for (auto& r : c->prof) {
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
    }
    c->prof.clear();
    if (c->prof_pending) cudaEventDestroy(c->prof_pending);
    c->prof_pending = nullptr;
}

}  // namespace spring

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

#define CTX_ENTER(ctx)                                                     \
    if (!(ctx)) return SPRING_ERR_ARG;                                      \
    DeviceGuard _guard((ctx)->device);                                      \
    (ctx)->err.clear()

int need(spring_ctx* c, bool ok, const char* what) {
    return ok ? SPRING_OK : fail(c, SPRING_ERR_STATE, "%s has not been set", what);
}

int set_temps(spring_ctx* c, const double* temps) {
    if (!temps) return fail(c, SPRING_ERR_ARG, "temps is NULL");
    for (int i = 0; i < c->nT; ++i)
        if (!(temps[i] > 0.0)) return fail(c, SPRING_ERR_ARG, "temperature %d is not positive", i + 1);
    // unchanged temperatures are not copied again
    if (c->d_temps.p && c->temps.size() == (size_t)c->nT && std::equal(temps, temps + c->nT, c->temps.begin()))
        return SPRING_OK;
    c->temps.assign(temps, temps + c->nT);
    SPRING_CHECK(dalloc(c, c->d_temps, c->nT, "temperatures"));
    return h2d(c, c->d_temps.p, temps, sizeof(double) * c->nT, "temperatures");
}

Pol make_pol(spring_ctx* c, const int* pol3) {
    Pol p;
    for (int k = 0; k < 3; ++k) {
        p.lo[k] = pol3 ? pol3[2 * k] - 1 : 0;
        p.hi[k] = pol3 ? pol3[2 * k + 1] - 1 : c->ndof - 1;
    }
    return p;
}

int check_pol(spring_ctx* c, const int* pol3) {
    if (!pol3) return SPRING_OK;
    for (int k = 0; k < 3; ++k)
        if (pol3[2 * k] < 1 || pol3[2 * k + 1] > c->ndof || pol3[2 * k] > pol3[2 * k + 1])
            return fail(c, SPRING_ERR_ARG, "pol3 column %d out of range [1,%d]", k + 1, c->ndof);
    return SPRING_OK;
}

int check_q0_range(spring_ctx* c, int i0_first, int n_q0) {
    if (!c->irr_set) return fail(c, SPRING_ERR_STATE, "irreducible q-points have not been set");
    if (n_q0 < 0 || i0_first < 1 || i0_first + n_q0 - 1 > c->nq0)
        return fail(c, SPRING_ERR_ARG, "q0 range [%d, %d] outside [1, %d]", i0_first, i0_first + n_q0 - 1, c->nq0);
    return SPRING_OK;
}

// Copy a [T][q0 range][s] device slab to the Fortran array out(Ndof, n_q0, nT).
int copy_lw_out(spring_ctx* c, const double* d_src, int q0_first, int n_q0, double* out) {
    if (!out) return SPRING_OK;
    for (int t = 0; t < c->nT; ++t)
        SPRING_CHECK(d2h(c, out + (size_t)t * n_q0 * c->ndof, d_src + ((size_t)t * c->nq0 + q0_first) * c->ndof,
                         sizeof(double) * n_q0 * c->ndof, "linewidth output"));
    return SPRING_OK;
}

}  // namespace

extern "C" {

int spring_ctx_create(spring_ctx** out, const spring_dims* d) {
    if (!out || !d) return SPRING_ERR_ARG;
    *out = nullptr;
    if (d->nbasis < 1 || d->nbasis > MAX_NB) return SPRING_ERR_ARG;
    if (d->mesh[0] < 1 || d->mesh[1] < 1 || d->mesh[2] < 1 || d->n_temps < 1) return SPRING_ERR_ARG;
    long long nq = (long long)d->mesh[0] * d->mesh[1] * d->mesh[2];
    if (nq > (1LL << 24)) return SPRING_ERR_ARG;
    spring_ctx* c = new (std::nothrow) spring_ctx();
    if (!c) return SPRING_ERR_ALLOC;
    if (d->device >= 0) {
        c->device = d->device;
    } else if (cudaGetDevice(&c->device) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return SPRING_ERR_CUDA;
    }
    DeviceGuard g(c->device);
    c->nb = d->nbasis;
    c->ndof = 3 * d->nbasis;
    for (int k = 0; k < 3; ++k) c->mesh[k] = d->mesh[k];
    c->nq = (int)nq;
    c->nT = d->n_temps;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return SPRING_ERR_CUDA;
    }
    c->stream = c->own_stream;
    *out = c;
    return SPRING_OK;
}

int spring_ctx_destroy(spring_ctx* c) {
    if (!c) return SPRING_ERR_ARG;
    {
        DeviceGuard g(c->device);
        cudaStreamSynchronize(c->stream);
        clear_profile(c);
        dfree(c->d_mass_rs); dfree(c->d_fc2); dfree(c->d_fc2_idx); dfree(c->d_fc2_num);
        dfree(c->d_fc4); dfree(c->d_fc4_posr); dfree(c->d_fc4_btyp); dfree(c->d_fc4_off);
        dfree(c->d_fc3); dfree(c->d_fc3_off); dfree(c->d_fc3_posr); dfree(c->d_fc3_btyp);
        dfree(c->d_qint); dfree(c->d_qpnt); dfree(c->d_tetra);
        dfree(c->d_tr_partner); dfree(c->d_tr_solve); dfree(c->d_tr_fill);
        dfree(c->d_irr_int); dfree(c->d_irr_q); dfree(c->d_mult); dfree(c->d_pos); dfree(c->d_temps);
        free_phonons(c->ph_grid); free_phonons(c->ph_irr);
        free_pairs(c->ps_irr); free_pairs(c->ps_tr);
        dfree(c->d_tr_int); dfree(c->d_tr_grid); dfree(c->d_tr_pos); dfree(c->d_tr_sgn); dfree(c->d_tr_deg);
        dfree(c->d_neg); dfree(c->d_wtr);
        dfree(c->d_bteg_row); dfree(c->d_bteg_kk); dfree(c->d_bteg_pq);
        dfree(c->ew.g); dfree(c->ew.r); dfree(c->ew.hz); dfree(c->ew.tau); dfree(c->ew.z); dfree(c->ew.cc);
        dfree(c->ew.dd); dfree(c->d_v4_rec);
        dfree(c->pd.vfc); dfree(c->pd.vm); dfree(c->pd.qpnt); dfree(c->pd.w2); dfree(c->pd.qint); dfree(c->pd.tet);
        dfree(c->pd.inc); dfree(c->pd.gamma0); dfree(c->pd.wgt); dfree(c->pd.G); dfree(c->pd.te0);
        free_phonons(c->pd.ph);
        dfree(c->d_tc_a); dfree(c->d_tc_b); dfree(c->d_tc_q0); dfree(c->d_tc_modes); dfree(c->d_tc_cnt_cta); dfree(c->d_scr_sum); dfree(c->d_kap_part); dfree(c->d_scr_rot); dfree(c->d_scr_map); dfree(c->d_tc_entries); dfree(c->d_tr_ev); dfree(c->d_tr_om); dfree(c->d_tr_ob);
        dfree(c->d_tc_rec); dfree(c->d_tc_tiles);
        free_mlp(c->mlp);
        dfree(c->d_scr_rep); dfree(c->d_tc_keys); dfree(c->d_tc_keys_s); dfree(c->d_tc_vals); dfree(c->d_tc_cnt);
        dfree(c->d_tc_seg); dfree(c->d_tc_ntl); dfree(c->d_tc_toff); dfree(c->d_tc_sort);
        dfree(c->d_scan_tmp); dfree(c->d_w); dfree(c->d_lw_all); dfree(c->d_lw_tmp); dfree(c->d_p3);
        dfree(c->d_kappa); dfree(c->d_krn); dfree(c->d_rxyz); dfree(c->d_wiso);
        free_enum4(c);
        dfree(c->d_v4_ph); dfree(c->d_v4_etab); dfree(c->d_v4_wf); dfree(c->d_v4_c); dfree(c->d_v4_map);
        dfree(c->d_v4_img); dfree(c->d_v4_cnt); dfree(c->d_v4_seg); dfree(c->d_v4_ntl); dfree(c->d_v4_toff);
        dfree(c->d_v4_stat); dfree(c->d_v4_tiles);
        if (c->h_pin) cudaFreeHost(c->h_pin);
        if (c->h_stage) cudaFreeHost(c->h_stage);
        if (c->ev_stage) cudaEventDestroy(c->ev_stage);
        if (c->ev_aux) cudaEventDestroy(c->ev_aux);
        if (c->ev_fork) cudaEventDestroy(c->ev_fork);
        if (c->ev_join) cudaEventDestroy(c->ev_join);
        if (c->stream2) cudaStreamDestroy(c->stream2);
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
    }
    delete c;
    return SPRING_OK;
}

const char* spring_last_error(const spring_ctx* c) { return c ? c->err.c_str() : "NULL context"; }

int spring_set_stream(spring_ctx* c, void* s) {
    CTX_ENTER(c);
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    return SPRING_OK;
}

int spring_synchronize(spring_ctx* c) {
    CTX_ENTER(c);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    return e == cudaSuccess ? SPRING_OK : cuda_fail(c, e, "synchronize");
}

int spring_kernel_launches(const spring_ctx* c, long long* count) {
    if (!c || !count) return SPRING_ERR_ARG;
    *count = c->launches;
    return SPRING_OK;
}

int spring_binary_version(int device, int* version) {
    if (!version) return SPRING_ERR_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    cudaFuncAttributes fa{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_sum2);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return SPRING_ERR_CUDA;
    }
    *version = fa.binaryVersion;
    return SPRING_OK;
}

int spring_tc_stats(const spring_ctx* c, int* n_tiles, int* n_pairs) {
    if (!c || !n_tiles || !n_pairs) return SPRING_ERR_ARG;
    const bool valid = c->tc_gen >= 0;
    *n_tiles = valid ? c->tc_ntiles : 0;
    *n_pairs = valid ? c->tc_npairs : 0;
    return SPRING_OK;
}

int spring_kappa_iter(spring_ctx* c, double eps_k, int max_iter, double* kappa, double* kappa_rta, int* iters) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->fc3_set, "FC3"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    if (!(eps_k > 0.0) || max_iter < 0) return fail(c, SPRING_ERR_ARG, "eps_k must be > 0 and max_iter >= 0");
    return run_bte(c, eps_k, max_iter, kappa, kappa_rta, iters);
}

int spring_kappa_iter_gauss(spring_ctx* c, double sigma, double eps_k, int max_iter, double* kappa, double* kappa_rta,
                            int* iters, double* stats) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->fc3_set, "FC3"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    if (!(eps_k > 0.0) || max_iter < 0) return fail(c, SPRING_ERR_ARG, "eps_k must be > 0 and max_iter >= 0");
    if (!(sigma > 0.0)) return fail(c, SPRING_ERR_ARG, "sigma must be > 0");
    return run_bte_gauss(c, sigma, eps_k, max_iter, kappa, kappa_rta, iters, stats);
}

int spring_set_option(spring_ctx* c, int option, int value) {
    CTX_ENTER(c);
    switch (option) {
        case SPRING_OPT_GENERIC_V3: c->force_generic_v3 = value != 0; return SPRING_OK;
        case SPRING_OPT_WAIT_POLLS: c->tc_max_spins = value < 0 ? -1 : (long long)value; return SPRING_OK;
        case SPRING_OPT_FP64_PRESCREEN: c->fp64_prescreen = value != 0; return SPRING_OK;
        default: return fail(c, SPRING_ERR_ARG, "unknown option %d", option);
    }
}

int spring_set_profiling(spring_ctx* c, int on) {
    CTX_ENTER(c);
    cudaStreamSynchronize(c->stream);
    clear_profile(c);
    c->profiling = on != 0;
    return SPRING_OK;
}

int spring_kernel_time(spring_ctx* c, const char* prefix, double* ms, long long* count) {
    CTX_ENTER(c);
    if (!prefix || !ms) return fail(c, SPRING_ERR_ARG, "prefix/ms is NULL");
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel_time");
    double tot = 0.0;
    long long n = 0;
    const size_t lp = std::strlen(prefix);
    for (auto& r : c->prof) {
        if (r.name.compare(0, lp, prefix) != 0) continue;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.start, r.stop) == cudaSuccess) {
            tot += t;
            ++n;
        }
    }
    *ms = tot;
    if (count) *count = n;
    return SPRING_OK;
}

int spring_prepare3(spring_ctx* c) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    c->ps_irr.n0 = c->nq0;
    c->ps_irr.q0_int = c->d_irr_int.p;
    return run_enumerate3(c, c->ps_irr);
}

int spring_debug_inject_fault(spring_ctx* c, int kind, int n) {
    CTX_ENTER(c);
    if (kind < 0 || kind > 2 || n < 0) return fail(c, SPRING_ERR_ARG, "kind must be 0..2 and n >= 0");
    c->inject_kind = n > 0 ? kind : -1;
    c->inject_n = n;
    for (int k = 0; k < 3; ++k) c->inject_seen[k] = 0;
    return SPRING_OK;
}

int spring_set_crystal(spring_ctx* c, const double* latvec, const double* mass) {
    CTX_ENTER(c);
    if (!latvec || !mass) return fail(c, SPRING_ERR_ARG, "latvec/mass is NULL");
    std::memcpy(c->latvec, latvec, sizeof c->latvec);
    const double* a = c->latvec;  // a[r + 3*i] = component r of vector i
    auto cross = [](const double* x, const double* y, double* o) {
        o[0] = x[1] * y[2] - x[2] * y[1];
        o[1] = x[2] * y[0] - x[0] * y[2];
        o[2] = x[0] * y[1] - x[1] * y[0];
    };
    double cr[3];
    cross(a + 3, a + 6, cr);
    c->vol = std::fabs(a[0] * cr[0] + a[1] * cr[1] + a[2] * cr[2]);
    if (!(c->vol > 0.0)) return fail(c, SPRING_ERR_ARG, "lattice vectors are degenerate");
    for (int i = 0; i < 3; ++i) {
        int i2 = (i + 1) % 3, i3 = (i + 2) % 3;
        cross(a + 3 * i2, a + 3 * i3, cr);
        for (int r = 0; r < 3; ++r) c->G[r + 3 * i] = cr[r] * 2.0 * (4.0 * std::atan(1.0)) / c->vol;
    }
    c->mass.assign(mass, mass + c->nb);
    std::vector<double> rs(c->nb);
    for (int i = 0; i < c->nb; ++i) {
        if (!(mass[i] > 0.0)) return fail(c, SPRING_ERR_ARG, "mass %d is not positive", i + 1);
        rs[i] = 1.0 / std::sqrt(mass[i]);
    }
    SPRING_CHECK(dalloc(c, c->d_mass_rs, c->nb, "masses"));
    SPRING_CHECK(h2d(c, c->d_mass_rs.p, rs.data(), sizeof(double) * c->nb, "masses"));
    c->crystal_set = true;
    return SPRING_OK;
}

int spring_set_dipole(spring_ctx* c, const double* atm_pos, const double* dielec, const double* born_z,
                      int decide_ew_param, double prec_ew, double lmb, const int* gmesh, const int* rmesh,
                      const int* sup_cell) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->crystal_set, "crystal"));
    return set_dipole(c, atm_pos, dielec, born_z, decide_ew_param, prec_ew, lmb, gmesh, rmesh, sup_cell);
}

int spring_set_point_defect(spring_ctx* c, const int* qmesh_pd, int na2_pd, const int* num_pd, const int* idx_pd,
                            const double* fc2_pd, const double* mass_def, double rho_def, int mat_inv_full,
                            int optc_therm) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->fc2_set, "FC2"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    return set_point_defect(c, qmesh_pd, na2_pd, num_pd, idx_pd, fc2_pd, mass_def, rho_def, mat_inv_full, optc_therm);
}

int spring_linewidth_pd(spring_ctx* c, int i0_first, int n_q0, double* rate, int add) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->pd.on, "point defect (spring_set_point_defect)"));
    SPRING_CHECK(need(c, c->ph_irr.set, "irreducible phonons"));
    if (i0_first < 1 || n_q0 < 0 || i0_first - 1 + n_q0 > c->nq0) return fail(c, SPRING_ERR_ARG, "q0 range out of bounds");
    if (n_q0 == 0) return SPRING_OK;
    const int q0 = i0_first - 1, n = c->ndof;
    DBuf<double> d_rate;
    SPRING_CHECK(dalloc(c, d_rate, (size_t)n_q0 * n, "point-defect rate"));
    int rc = run_point_defect(c, q0, n_q0, d_rate.p);
    if (rc == SPRING_OK && add) rc = run_point_defect_add(c, q0, n_q0, d_rate.p);
    if (rc == SPRING_OK && rate) rc = d2h(c, rate, d_rate.p, sizeof(double) * n_q0 * n, "point-defect rate");
    cudaStreamSynchronize(c->stream);
    dfree(d_rate);
    return rc;
}

int spring_get_dipole(spring_ctx* c, int* on, double* lmb, int* gmesh, int* n_r, int* n_g) {
    CTX_ENTER(c);
    if (on) *on = c->ew.on ? 1 : 0;
    if (lmb) *lmb = c->ew.lmb;
    if (gmesh)
        for (int k = 0; k < 3; ++k) gmesh[k] = c->ew.gmesh[k];
    if (n_r) *n_r = c->ew.nr;
    if (n_g) *n_g = c->ew.ng;
    return SPRING_OK;
}

int spring_set_fc2(spring_ctx* c, int na2, const int* num, const int* idx, const double* fc) {
    CTX_ENTER(c);
    if (!num || !idx || !fc || na2 < 1) return fail(c, SPRING_ERR_ARG, "FC2 arrays are NULL or na2 < 1");
    for (int mu = 0; mu < c->nb; ++mu) {
        if (num[mu] < 0 || num[mu] > na2) return fail(c, SPRING_ERR_ARG, "FC2 atm_num(%d) out of range", mu + 1);
        for (int n = 0; n < num[mu]; ++n) {
            int b = idx[4 * (n + (size_t)na2 * mu) + 3];
            if (b < 1 || b > c->nb) return fail(c, SPRING_ERR_ARG, "FC2 atm_indx basis out of range");
        }
    }
    c->na2 = na2;
    SPRING_CHECK(dalloc(c, c->d_fc2, (size_t)c->nb * na2 * 9, "FC2"));
    SPRING_CHECK(dalloc(c, c->d_fc2_idx, (size_t)c->nb * na2 * 4, "FC2 index"));
    SPRING_CHECK(dalloc(c, c->d_fc2_num, c->nb, "FC2 counts"));
    SPRING_CHECK(h2d(c, c->d_fc2.p, fc, sizeof(double) * c->nb * na2 * 9, "FC2"));
    SPRING_CHECK(h2d(c, c->d_fc2_idx.p, idx, sizeof(int) * c->nb * na2 * 4, "FC2 index"));
    SPRING_CHECK(h2d(c, c->d_fc2_num.p, num, sizeof(int) * c->nb, "FC2 counts"));
    c->h_fc2.assign(fc, fc + (size_t)c->nb * na2 * 9);
    c->h_fc2_idx.assign(idx, idx + (size_t)c->nb * na2 * 4);
    c->h_fc2_num.assign(num, num + c->nb);
    c->fc2_set = true;
    return SPRING_OK;
}

int spring_set_fc3(spring_ctx* c, int na3, const int* num, const int* idx, const double* fc) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->crystal_set, "crystal"));
    if (!num || !idx || !fc || na3 < 1 || na3 > 16) return fail(c, SPRING_ERR_ARG, "FC3 arrays are NULL or na3 not in 1..16");
    const int nb = c->nb;
    // kernel layout: [mu][k2 = N2*3+gamma][r = (N1*3+alpha)*3+beta], zero padded beyond atm_num
    // Device layout [mu][N1][N2][alpha][beta][gamma] (the Fortran memory order), zero beyond
    // atm_num, with the neighbour slots of each mu reordered so that slots of the same basis
    // atom are contiguous (stable); off[mu][nu] .. off[mu][nu+1] are the slots of basis nu.
    // Only the order of the sums over N1/N2 changes.
    std::vector<double> t((size_t)nb * na3 * na3 * 27, 0.0), posr((size_t)nb * na3 * 3, 0.0);
    std::vector<int> btyp((size_t)nb * na3, 0), off((size_t)nb * (nb + 1), 0);
    for (int mu = 0; mu < nb; ++mu) {
        if (num[mu] < 0 || num[mu] > na3) return fail(c, SPRING_ERR_ARG, "FC3 atm_num(%d) out of range", mu + 1);
        std::vector<int> order;  // new slot -> original slot
        for (int nu = 0; nu < nb; ++nu) {
            off[(size_t)mu * (nb + 1) + nu] = (int)order.size();
            for (int n = 0; n < num[mu]; ++n) {
                const int* e = idx + 4 * (n + (size_t)na3 * mu);
                if (e[3] < 1 || e[3] > nb) return fail(c, SPRING_ERR_ARG, "FC3 atm_indx basis out of range");
                if (e[3] - 1 == nu) order.push_back(n);
            }
        }
        off[(size_t)mu * (nb + 1) + nb] = (int)order.size();
        for (int k = 0; k < num[mu]; ++k) {
            const int n = order[k];
            const int* e = idx + 4 * (n + (size_t)na3 * mu);
            btyp[(size_t)mu * na3 + k] = e[3] - 1;
            for (int r = 0; r < 3; ++r)  // atmPosR = latvec * cell (FC3_mod.f90:84)
                posr[((size_t)mu * na3 + k) * 3 + r] =
                    c->latvec[r] * e[0] + c->latvec[r + 3] * e[1] + c->latvec[r + 6] * e[2];
        }
        for (int k1 = 0; k1 < num[mu]; ++k1)
            for (int k2 = 0; k2 < num[mu]; ++k2)
                for (int abc = 0; abc < 27; ++abc) {
                    // Fortran fC(ga,be,al,N2,N1,mu): abc = (al*3+be)*3+ga is the fastest index
                    const int n1 = order[k1], n2 = order[k2];
                    t[((size_t)(mu * na3 + k1) * na3 + k2) * 27 + abc] =
                        fc[((size_t)(mu * na3 + n1) * na3 + n2) * 27 + abc];
                }
    }
    c->na3 = na3;
    SPRING_CHECK(dalloc(c, c->d_fc3_off, off.size(), "FC3 slot offsets"));
    SPRING_CHECK(h2d(c, c->d_fc3_off.p, off.data(), sizeof(int) * off.size(), "FC3 slot offsets"));
    SPRING_CHECK(dalloc(c, c->d_fc3, t.size(), "FC3"));
    SPRING_CHECK(dalloc(c, c->d_fc3_posr, posr.size(), "FC3 positions"));
    SPRING_CHECK(dalloc(c, c->d_fc3_btyp, btyp.size(), "FC3 basis"));
    SPRING_CHECK(h2d(c, c->d_fc3.p, t.data(), sizeof(double) * t.size(), "FC3"));
    SPRING_CHECK(h2d(c, c->d_fc3_posr.p, posr.data(), sizeof(double) * posr.size(), "FC3 positions"));
    SPRING_CHECK(h2d(c, c->d_fc3_btyp.p, btyp.data(), sizeof(int) * btyp.size(), "FC3 basis"));
    // no stream wait: h2d staged every byte in the context's pinned ring before queuing its copy
    c->fc3_set = true;
    dfree(c->d_wtr);  // cached W grids depend on FC3
    c->bteg_n = 0;    // and so does the Gaussian BTE operator
    return SPRING_OK;
}

int spring_set_fc4(spring_ctx* c, int na4, const int* num, const int* idx, const double* fc) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->crystal_set, "crystal"));
    if (!num || !idx || !fc || na4 < 1 || na4 > 16) return fail(c, SPRING_ERR_ARG, "FC4 arrays are NULL or na4 not in 1..16");
    const int nb = c->nb;
    const size_t blk = 81;
    std::vector<double> t((size_t)nb * na4 * na4 * na4 * blk, 0.0), posr((size_t)nb * na4 * 3, 0.0);
    std::vector<int> btyp((size_t)nb * na4, 0), off((size_t)nb * (nb + 1), 0);
    for (int mu = 0; mu < nb; ++mu) {
        if (num[mu] < 0 || num[mu] > na4) return fail(c, SPRING_ERR_ARG, "FC4 atm_num(%d) out of range", mu + 1);
        std::vector<int> order;  // slots grouped by basis atom (stable), as for FC3
        for (int nu = 0; nu < nb; ++nu) {
            off[(size_t)mu * (nb + 1) + nu] = (int)order.size();
            for (int n = 0; n < num[mu]; ++n) {
                const int* e = idx + 4 * (n + (size_t)na4 * mu);
                if (e[3] < 1 || e[3] > nb) return fail(c, SPRING_ERR_ARG, "FC4 atm_indx basis out of range");
                if (e[3] - 1 == nu) order.push_back(n);
            }
        }
        off[(size_t)mu * (nb + 1) + nb] = (int)order.size();
        for (int k = 0; k < num[mu]; ++k) {
            const int* e = idx + 4 * (order[k] + (size_t)na4 * mu);
            btyp[(size_t)mu * na4 + k] = e[3] - 1;
            for (int r = 0; r < 3; ++r)  // atmPosR = latvec * cell (FC4_mod.f90:74-93)
                posr[((size_t)mu * na4 + k) * 3 + r] =
                    c->latvec[r] * e[0] + c->latvec[r + 3] * e[1] + c->latvec[r + 6] * e[2];
        }
        for (int k1 = 0; k1 < num[mu]; ++k1)
            for (int k2 = 0; k2 < num[mu]; ++k2)
                for (int k3 = 0; k3 < num[mu]; ++k3) {
                    const size_t dst = (((size_t)(mu * na4 + k1) * na4 + k2) * na4 + k3) * blk;
                    const size_t src = (((size_t)(mu * na4 + order[k1]) * na4 + order[k2]) * na4 + order[k3]) * blk;
                    for (size_t x = 0; x < blk; ++x) t[dst + x] = fc[src + x];
                }
    }
    c->na4 = na4;
    SPRING_CHECK(dalloc(c, c->d_fc4, t.size(), "FC4"));
    SPRING_CHECK(dalloc(c, c->d_fc4_posr, posr.size(), "FC4 positions"));
    SPRING_CHECK(dalloc(c, c->d_fc4_btyp, btyp.size(), "FC4 basis"));
    SPRING_CHECK(dalloc(c, c->d_fc4_off, off.size(), "FC4 slot offsets"));
    SPRING_CHECK(h2d(c, c->d_fc4.p, t.data(), sizeof(double) * t.size(), "FC4"));
    SPRING_CHECK(h2d(c, c->d_fc4_posr.p, posr.data(), sizeof(double) * posr.size(), "FC4 positions"));
    SPRING_CHECK(h2d(c, c->d_fc4_btyp.p, btyp.data(), sizeof(int) * btyp.size(), "FC4 basis"));
    SPRING_CHECK(h2d(c, c->d_fc4_off.p, off.data(), sizeof(int) * off.size(), "FC4 slot offsets"));
    // no stream wait: h2d staged every byte in the context's pinned ring before queuing its copy
    c->fc4_set = true;
    return SPRING_OK;
}

int spring_make_mesh(spring_ctx* c, const int* shift, int zero_centered, int* q_pnt_int, double* q_pnt,
                     int* tetrahedrons) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->crystal_set, "crystal"));
    int sh[3] = {0, 0, 0};
    if (shift) for (int k = 0; k < 3; ++k) sh[k] = shift[k];
    const size_t nq = c->nq;
    SPRING_CHECK(dalloc(c, c->d_qint, nq * 3, "q_pnt_int"));
    SPRING_CHECK(dalloc(c, c->d_qpnt, nq * 3, "q_pnt"));
    SPRING_CHECK(dalloc(c, c->d_tetra, nq * 24, "tetrahedrons"));
    SPRING_CHECK(run_make_mesh(c, sh, zero_centered));
    if (q_pnt_int) SPRING_CHECK(d2h(c, q_pnt_int, c->d_qint.p, sizeof(int) * nq * 3, "q_pnt_int"));
    if (q_pnt) SPRING_CHECK(d2h(c, q_pnt, c->d_qpnt.p, sizeof(double) * nq * 3, "q_pnt"));
    if (tetrahedrons) {
        std::vector<int> t(nq * 24);
        SPRING_CHECK(d2h(c, t.data(), c->d_tetra.p, sizeof(int) * nq * 24, "tetrahedrons"));
        for (size_t i = 0; i < t.size(); ++i) tetrahedrons[i] = t[i] + 1;
    }
    // no stream wait: the mesh kernels are queued like any other, and each requested readback waits
    c->mesh_set = true;
    c->mesh_zc = zero_centered != 0;
    // the time-reversal lists depend only on the mesh dimensions (fixed per context): kept
    for (int k = 0; k < 3; ++k) c->mesh_shift[k] = sh[k];
    c->ps_irr.done = false;
    c->ps_tr.done = false;
    c->ntr = 0;
    return SPRING_OK;
}

static int install_irr(spring_ctx* c, int nq0, const int* irr_int, const int* pos, const int* mult) {
    c->nq0 = nq0;
    c->h_irr_int.assign(irr_int, irr_int + 3 * nq0);
    c->h_pos.assign(pos, pos + c->nq);
    c->h_mult.assign(mult, mult + nq0);
    std::vector<double> q((size_t)nq0 * 3);
    for (int i = 0; i < nq0; ++i)
        for (int r = 0; r < 3; ++r) {
            double s = 0.0;  // Recp_cell_unit * irr (TetrahedronQ_m.f90:304)
            for (int k = 0; k < 3; ++k) s += (c->G[r + 3 * k] / c->mesh[k]) * double(irr_int[3 * i + k]);
            q[3 * i + r] = s;
        }
    SPRING_CHECK(dalloc(c, c->d_irr_int, (size_t)nq0 * 3, "irreducible q"));
    SPRING_CHECK(dalloc(c, c->d_irr_q, (size_t)nq0 * 3, "irreducible q"));
    SPRING_CHECK(dalloc(c, c->d_mult, nq0, "multiplicity"));
    SPRING_CHECK(h2d(c, c->d_irr_int.p, irr_int, sizeof(int) * nq0 * 3, "irreducible q"));
    SPRING_CHECK(h2d(c, c->d_irr_q.p, q.data(), sizeof(double) * nq0 * 3, "irreducible q"));
    SPRING_CHECK(h2d(c, c->d_mult.p, mult, sizeof(int) * nq0, "multiplicity"));
    SPRING_CHECK(dalloc(c, c->d_pos, c->nq, "pos"));
    SPRING_CHECK(h2d(c, c->d_pos.p, pos, sizeof(int) * c->nq, "pos"));
    SPRING_CHECK(dalloc(c, c->d_lw_all, (size_t)c->nT * nq0 * c->ndof, "LW_Allq0"));
    SPRING_CHECK(zero(c, c->d_lw_all.p, sizeof(double) * c->nT * nq0 * c->ndof, "LW_Allq0"));
    // no stream wait: h2d staged every byte in the context's pinned ring before queuing its copy
    c->irr_set = true;
    c->ps_irr.done = false;
    c->ps_irr.n0 = nq0;
    c->ps_irr.q0_int = c->d_irr_int.p;
    c->ph_irr.set = false;  // buffers kept; recomputed for the new set
    return SPRING_OK;
}

int spring_find_irr_q(spring_ctx* c, int nrot, const int* rot, int time_rev, int* nq0_out, int* irr_q_pnt_int,
                      int* pos, int* multiplicity) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    if (nrot < 1 || nrot > 192 || !rot) return fail(c, SPRING_ERR_ARG, "rotations: need 1..192 matrices");
    DBuf<int>&d_rot = c->d_scr_rot, &d_map = c->d_scr_map;  // kept between calls
    int rc = dalloc(c, d_rot, (size_t)nrot * 9, "rotations");
    if (rc == SPRING_OK) rc = dalloc(c, d_map, c->nq, "irreducible map");
    if (rc == SPRING_OK) rc = h2d(c, d_rot.p, rot, sizeof(int) * 9 * nrot, "rotations");
    if (rc == SPRING_OK) rc = run_irr_map(c, d_rot.p, nrot, time_rev, d_map.p);
    std::vector<int> map(c->nq), qint((size_t)c->nq * 3);
    if (rc == SPRING_OK) rc = d2h(c, map.data(), d_map.p, sizeof(int) * c->nq, "irreducible map");
    if (rc == SPRING_OK) rc = d2h(c, qint.data(), c->d_qint.p, sizeof(int) * c->nq * 3, "q_pnt_int");
    if (rc != SPRING_OK) return rc;
    // unique_sort + FindPositionAndMultiplicity (Helper_m.f90:510-594): the representatives are grid
    // indices, so their ascending order and ranks come from one pass over a flag array.
    std::vector<int> rank(c->nq, -1);
    for (int i = 0; i < c->nq; ++i) {
        if (map[i] < 0 || map[i] >= c->nq) return fail(c, SPRING_ERR_CUDA, "irreducible map out of range");
        rank[map[i]] = 0;
    }
    int nq0 = 0;
    for (int g = 0; g < c->nq; ++g)
        if (rank[g] == 0) rank[g] = ++nq0;  // 1-based position
    std::vector<int> irr((size_t)nq0 * 3), ps(c->nq), mu(nq0, 0);
    for (int g = 0; g < c->nq; ++g)
        if (rank[g] > 0)
            for (int d = 0; d < 3; ++d) irr[3 * (rank[g] - 1) + d] = qint[3 * (size_t)g + d];
    for (int i = 0; i < c->nq; ++i) {
        ps[i] = rank[map[i]];
        mu[ps[i] - 1] += 1;
    }
    SPRING_CHECK(install_irr(c, nq0, irr.data(), ps.data(), mu.data()));
    if (nq0_out) *nq0_out = nq0;
    if (irr_q_pnt_int) std::memcpy(irr_q_pnt_int, irr.data(), sizeof(int) * irr.size());
    if (pos) std::memcpy(pos, ps.data(), sizeof(int) * ps.size());
    if (multiplicity) std::memcpy(multiplicity, mu.data(), sizeof(int) * mu.size());
    return SPRING_OK;
}

int spring_compute_phonons(spring_ctx* c, const double* temps, double freq_cut) {
    CTX_ENTER(c);
    (void)freq_cut;
    SPRING_CHECK(need(c, c->fc2_set, "FC2"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    SPRING_CHECK(set_temps(c, temps));
    SPRING_CHECK(alloc_phonons(c, c->ph_grid, c->nq));
    SPRING_CHECK(alloc_phonons(c, c->ph_irr, c->nq0));
    SPRING_CHECK(run_phonons_mesh(c));
    c->ph_grid.set = c->ph_irr.set = true;
    c->ph_gen += 1;
    dfree(c->d_wtr);  // cached W grids depend on the phonons
    return SPRING_OK;
}

int spring_set_phonons(spring_ctx* c, int which, const double* temps, const double* evec, const double* omega,
                       const double* oneby, const double* nbe, const double* vel) {
    CTX_ENTER(c);
    if (which == 2) {  // the point-defect mesh: eigenvectors and omegas only
        SPRING_CHECK(need(c, c->pd.on, "point defect (spring_set_point_defect)"));
        if (!evec || !omega) return fail(c, SPRING_ERR_ARG, "phonon arrays are NULL");
        const size_t nd = c->ndof, n = c->pd.nq;
        SPRING_CHECK(h2d(c, c->pd.ph.evec.p, evec, sizeof(double2) * n * nd * nd, "eigenvectors"));
        SPRING_CHECK(h2d(c, c->pd.ph.omega.p, omega, sizeof(double) * n * nd, "omega"));
        return SPRING_OK;
    }
    if (which != 0 && which != 1) return fail(c, SPRING_ERR_ARG, "which must be 0 (grid), 1 (irreducible) or 2");
    if (!evec || !omega || !oneby || !nbe || !vel) return fail(c, SPRING_ERR_ARG, "phonon arrays are NULL");
    if (which == 1) SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    SPRING_CHECK(set_temps(c, temps));
    Phonons& p = which == 0 ? c->ph_grid : c->ph_irr;
    const int n = which == 0 ? c->nq : c->nq0;
    SPRING_CHECK(alloc_phonons(c, p, n));
    const size_t nd = c->ndof;
    SPRING_CHECK(h2d(c, p.evec.p, evec, sizeof(double2) * n * nd * nd, "eigenvectors"));
    SPRING_CHECK(h2d(c, p.omega.p, omega, sizeof(double) * n * nd, "omega"));
    SPRING_CHECK(h2d(c, p.oneby.p, oneby, sizeof(double) * n * nd, "1/omega"));
    SPRING_CHECK(h2d(c, p.nbe.p, nbe, sizeof(double) * c->nT * n * nd, "nBE"));
    SPRING_CHECK(h2d(c, p.vel.p, vel, sizeof(double) * n * nd * 3, "group velocity"));
    p.set = true;
    c->ph_gen += 1;
    if (which == 0) dfree(c->d_wtr);  // cached W grids depend on the grid phonons
    return SPRING_OK;
}

int spring_get_phonons(spring_ctx* c, int which, double* evec, double* omega, double* oneby, double* nbe,
                       double* vel) {
    CTX_ENTER(c);
    if (which == 2) SPRING_CHECK(need(c, c->pd.on, "point defect (spring_set_point_defect)"));
    if (which < 0 || which > 2) return fail(c, SPRING_ERR_ARG, "which must be 0, 1 or 2");
    Phonons& p = which == 0 ? c->ph_grid : (which == 1 ? c->ph_irr : c->pd.ph);
    if (which == 2) {
        const size_t nd = c->ndof, n = c->pd.nq;
        if (evec) SPRING_CHECK(d2h(c, evec, p.evec.p, sizeof(double2) * n * nd * nd, "eigenvectors"));
        if (omega) SPRING_CHECK(d2h(c, omega, p.omega.p, sizeof(double) * n * nd, "omega"));
        return SPRING_OK;
    }
    SPRING_CHECK(need(c, p.set, "phonons"));
    const size_t nd = c->ndof, n = p.n;
    if (evec) SPRING_CHECK(d2h(c, evec, p.evec.p, sizeof(double2) * n * nd * nd, "eigenvectors"));
    if (omega) SPRING_CHECK(d2h(c, omega, p.omega.p, sizeof(double) * n * nd, "omega"));
    if (oneby) SPRING_CHECK(d2h(c, oneby, p.oneby.p, sizeof(double) * n * nd, "1/omega"));
    if (nbe) SPRING_CHECK(d2h(c, nbe, p.nbe.p, sizeof(double) * c->nT * n * nd, "nBE"));
    if (vel) SPRING_CHECK(d2h(c, vel, p.vel.p, sizeof(double) * n * nd * 3, "group velocity"));
    return SPRING_OK;
}

int spring_enumerate3(spring_ctx* c, int i0, int* allq1q2, int* perm, int* counts) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0, 1));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    DBuf<int> a, p, n;
    int rc = dalloc(c, a, (size_t)c->nq * 4, "Allq1q2");
    if (rc == SPRING_OK) rc = dalloc(c, p, (size_t)c->nq * 2, "q1q2_permuted");
    if (rc == SPRING_OK) rc = dalloc(c, n, 2, "counts");
    if (rc == SPRING_OK) rc = run_enumerate3_fortran(c, i0 - 1, a.p, p.p, n.p);
    int hc[2] = {0, 0};
    if (rc == SPRING_OK) rc = d2h(c, hc, n.p, sizeof hc, "counts");
    if (rc == SPRING_OK && allq1q2) rc = d2h(c, allq1q2, a.p, sizeof(int) * 4 * c->nq, "Allq1q2");
    if (rc == SPRING_OK && perm) rc = d2h(c, perm, p.p, sizeof(int) * 2 * hc[0], "q1q2_permuted");
    if (rc == SPRING_OK && counts) { counts[0] = hc[0]; counts[1] = hc[1]; }
    dfree(a); dfree(p); dfree(n);
    return rc;
}

static int ensure_enum3(spring_ctx* c) {
    if (c->ps_irr.done) return SPRING_OK;
    c->ps_irr.n0 = c->nq0;
    c->ps_irr.q0_int = c->d_irr_int.p;
    return run_enumerate3(c, c->ps_irr);
}

static int ready3(spring_ctx* c) {
    SPRING_CHECK(need(c, c->fc3_set, "FC3"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    SPRING_CHECK(need(c, c->ph_irr.set, "irreducible-point phonons"));
    return SPRING_OK;
}

// Number of q0 whose W grids fit the tetrahedron W buffer (keeps it around L2 size).
static int w_slots(spring_ctx* c, int n_q0) {
    const size_t slot = (size_t)c->nq * c->ndof * c->ndof * c->ndof * sizeof(double);
    size_t budget = (size_t)96 << 20;
    int s = (int)std::max<size_t>(1, budget / slot);
    return std::min(s, std::max(n_q0, 1));
}

int spring_scatter_w3(spring_ctx* c, int i0, double* sctr) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0, 1));
    SPRING_CHECK(ready3(c));
    SPRING_CHECK(ensure_enum3(c));
    const size_t n = (size_t)c->nq * c->ndof * c->ndof * c->ndof;
    SPRING_CHECK(dalloc(c, c->d_w, n, "W buffer"));
    SPRING_CHECK(run_v3_wgrid(c, c->ps_irr, irr_view(c), i0 - 1, 1, c->d_w.p));
    if (sctr) SPRING_CHECK(d2h(c, sctr, c->d_w.p, sizeof(double) * n, "Sctrq1"));
    return SPRING_OK;
}

int spring_linewidth3(spring_ctx* c, int i0_first, int n_q0, int delta_mode, double sigma, const int* pol3,
                      double* lw, double* p3_q0) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0_first, n_q0));
    SPRING_CHECK(ready3(c));
    SPRING_CHECK(check_pol(c, pol3));
    if (delta_mode != SPRING_DELTA_GAUSS && delta_mode != SPRING_DELTA_TETRA)
        return fail(c, SPRING_ERR_ARG, "delta_mode must be SPRING_DELTA_GAUSS or SPRING_DELTA_TETRA");
    if (delta_mode == SPRING_DELTA_GAUSS && !(sigma > 0.0)) return fail(c, SPRING_ERR_ARG, "sigma must be > 0");
    if (n_q0 == 0) return SPRING_OK;
    SPRING_CHECK(ensure_enum3(c));
    const Pol pol = make_pol(c, pol3);
    const int q0 = i0_first - 1;
    const size_t nl = (size_t)c->nT * c->nq0 * c->ndof;
    SPRING_CHECK(dalloc(c, c->d_lw_tmp, nl, "linewidth scratch"));
    SPRING_CHECK(dalloc(c, c->d_p3, (size_t)c->nq0 * c->ndof, "phase-space scratch"));
    SPRING_CHECK(zero(c, c->d_lw_tmp.p, sizeof(double) * nl, "linewidth scratch"));
    SPRING_CHECK(zero(c, c->d_p3.p, sizeof(double) * c->nq0 * c->ndof, "phase-space scratch"));
    if (delta_mode == SPRING_DELTA_GAUSS) {
        SPRING_CHECK(run_v3_gauss(c, q0, n_q0, sigma, pol, c->d_lw_tmp.p, c->d_p3.p));
    } else {
        const int slots = w_slots(c, n_q0);
        const size_t slot = (size_t)c->nq * c->ndof * c->ndof * c->ndof;
        SPRING_CHECK(dalloc(c, c->d_w, slot * slots, "W buffer"));
        for (int b = 0; b < n_q0; b += slots) {
            const int nb = std::min(slots, n_q0 - b);
            SPRING_CHECK(run_v3_wgrid(c, c->ps_irr, irr_view(c), q0 + b, nb, c->d_w.p));
            SPRING_CHECK(run_tetra3(c, q0 + b, nb, c->d_w.p, pol, c->d_lw_tmp.p, c->d_p3.p));
        }
    }
    // LW_Allq0 += lw (third order: weight 1, main.f90:584)
    SPRING_CHECK(run_axpy_lw(c, 1.0, c->d_lw_tmp.p, c->d_lw_all.p, q0, n_q0));
    SPRING_CHECK(copy_lw_out(c, c->d_lw_tmp.p, q0, n_q0, lw));
    if (p3_q0)
        SPRING_CHECK(d2h(c, p3_q0, c->d_p3.p + (size_t)q0 * c->ndof, sizeof(double) * n_q0 * c->ndof, "P3_q0"));
    return SPRING_OK;
}

int spring_linewidth_iso(spring_ctx* c, int i0_first, int n_q0, int delta_mode, double sigma, const double* g2,
                         double* rate) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0_first, n_q0));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set && c->ph_irr.set, "phonons"));
    if (!g2) return fail(c, SPRING_ERR_ARG, "g2 is NULL");
    if (delta_mode != SPRING_DELTA_GAUSS && delta_mode != SPRING_DELTA_TETRA)
        return fail(c, SPRING_ERR_ARG, "delta_mode must be SPRING_DELTA_GAUSS or SPRING_DELTA_TETRA");
    if (delta_mode == SPRING_DELTA_GAUSS && !(sigma > 0.0)) return fail(c, SPRING_ERR_ARG, "sigma must be > 0");
    if (n_q0 == 0) return SPRING_OK;
    const int q0 = i0_first - 1;
    const size_t nl = (size_t)c->nT * c->nq0 * c->ndof;
    SPRING_CHECK(dalloc(c, c->d_lw_tmp, nl, "linewidth scratch"));
    SPRING_CHECK(zero(c, c->d_lw_tmp.p, sizeof(double) * nl, "linewidth scratch"));
    SPRING_CHECK(run_iso(c, q0, n_q0, delta_mode, sigma, g2, c->d_lw_tmp.p));
    SPRING_CHECK(run_axpy_lw(c, 0.5, c->d_lw_tmp.p, c->d_lw_all.p, q0, n_q0));
    SPRING_CHECK(copy_lw_out(c, c->d_lw_tmp.p, q0, n_q0, rate));
    return SPRING_OK;
}

int spring_enumerate4(spring_ctx* c, int i0, int* allq1q2q3, int* perm, long long cap, long long* counts) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0, 1));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    if (perm && cap < 0) return fail(c, SPRING_ERR_ARG, "cap must be >= 0");
    const size_t cells = (size_t)c->nq * c->nq;
    DBuf<int> a, p;
    long long hc[2] = {0, 0};
    int rc = SPRING_OK;
    if (allq1q2q3) rc = dalloc(c, a, cells * 3, "Allq1q2q3");
    if (rc == SPRING_OK && perm) rc = dalloc(c, p, (size_t)std::max<long long>(cap, 1) * 3, "q1q2q3_permuted");
    if (rc == SPRING_OK) rc = run_enumerate4_fortran(c, i0 - 1, a.p, p.p, cap, hc);
    if (rc == SPRING_OK && perm && hc[0] > cap)
        rc = fail(c, SPRING_ERR_ARG, "%lld quartets exceed cap = %lld", hc[0], cap);
    if (rc == SPRING_OK && allq1q2q3) rc = d2h(c, allq1q2q3, a.p, sizeof(int) * 3 * cells, "Allq1q2q3");
    if (rc == SPRING_OK && perm) rc = d2h(c, perm, p.p, sizeof(int) * 3 * (size_t)hc[0], "q1q2q3_permuted");
    if (rc == SPRING_OK && counts) { counts[0] = hc[0]; counts[1] = hc[1]; }
    dfree(a); dfree(p);
    return rc;
}

int spring_linewidth4(spring_ctx* c, int i0_first, int n_q0, int delta_mode, double sigma, const int* pol4,
                      double* rate) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0_first, n_q0));
    SPRING_CHECK(need(c, c->fc4_set, "FC4"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    SPRING_CHECK(need(c, c->ph_irr.set, "irreducible-point phonons"));
    if (delta_mode != SPRING_DELTA_GAUSS && delta_mode != SPRING_DELTA_TETRA)
        return fail(c, SPRING_ERR_ARG, "delta_mode must be SPRING_DELTA_GAUSS or SPRING_DELTA_TETRA");
    if (delta_mode == SPRING_DELTA_GAUSS && !(sigma > 0.0)) return fail(c, SPRING_ERR_ARG, "sigma must be > 0");
    if (pol4)
        for (int k = 0; k < 4; ++k)
            if (pol4[2 * k] < 1 || pol4[2 * k + 1] > c->ndof || pol4[2 * k] > pol4[2 * k + 1])
                return fail(c, SPRING_ERR_ARG, "pol4 column %d outside 1..Ndof", k + 1);
    if (n_q0 == 0) return SPRING_OK;
    const int q0 = i0_first - 1;
    const size_t nl = (size_t)c->nT * c->nq0 * c->ndof;
    SPRING_CHECK(dalloc(c, c->d_lw_tmp, nl, "linewidth scratch"));
    SPRING_CHECK(zero(c, c->d_lw_tmp.p, sizeof(double) * nl, "linewidth scratch"));
    // Tensor cores (spring_set_precision BF16 / BF16x3) for the Gaussian rate of two-atom cells over
    // every branch; otherwise (and for the tetrahedron form) the FP64 kernels.
    bool handled = false;
    bool all_modes = true;
    if (pol4)
        for (int k = 0; k < 4; ++k) all_modes = all_modes && pol4[2 * k] == 1 && pol4[2 * k + 1] == c->ndof;
    if (delta_mode == SPRING_DELTA_GAUSS && all_modes)
        SPRING_CHECK(run_v4tc_gauss(c, q0, n_q0, sigma, nullptr, c->d_lw_tmp.p, &handled));
    if (!handled) SPRING_CHECK(run_lw4(c, q0, n_q0, delta_mode, sigma, pol4, c->d_lw_tmp.p));
    SPRING_CHECK(run_axpy_lw(c, 0.5, c->d_lw_tmp.p, c->d_lw_all.p, q0, n_q0));
    SPRING_CHECK(copy_lw_out(c, c->d_lw_tmp.p, q0, n_q0, rate));
    return SPRING_OK;
}

int spring_linewidth4_modes(spring_ctx* c, int i0_first, int n_q0, double sigma, const int* s0_mask, double* rate) {
    CTX_ENTER(c);
    SPRING_CHECK(check_q0_range(c, i0_first, n_q0));
    SPRING_CHECK(need(c, c->fc4_set, "FC4"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    SPRING_CHECK(need(c, c->ph_irr.set, "irreducible-point phonons"));
    if (!s0_mask || !rate) return fail(c, SPRING_ERR_ARG, "s0_mask and rate must not be NULL");
    if (!(sigma > 0.0)) return fail(c, SPRING_ERR_ARG, "sigma must be > 0");
    const int full = (1 << c->ndof) - 1;
    for (int k = 0; k < n_q0; ++k)
        if (s0_mask[k] & ~full) return fail(c, SPRING_ERR_ARG, "s0_mask(%d) has bits beyond Ndof", k + 1);
    if (n_q0 == 0) return SPRING_OK;
    const int q0 = i0_first - 1;
    const size_t nl = (size_t)c->nT * c->nq0 * c->ndof;
    SPRING_CHECK(dalloc(c, c->d_lw_tmp, nl, "linewidth scratch"));
    SPRING_CHECK(zero(c, c->d_lw_tmp.p, sizeof(double) * nl, "linewidth scratch"));
    bool handled = false;
    SPRING_CHECK(run_v4tc_gauss(c, q0, n_q0, sigma, s0_mask, c->d_lw_tmp.p, &handled));
    if (!handled) SPRING_CHECK(run_lw4(c, q0, n_q0, SPRING_DELTA_GAUSS, sigma, nullptr, c->d_lw_tmp.p));
    SPRING_CHECK(copy_lw_out(c, c->d_lw_tmp.p, q0, n_q0, rate));
    // branches outside the mask are zero (the FP64 path computes every branch)
    for (int T = 0; T < c->nT; ++T)
        for (int k = 0; k < n_q0; ++k)
            for (int s = 0; s < c->ndof; ++s)
                if (!((s0_mask[k] >> s) & 1)) rate[((size_t)T * n_q0 + k) * c->ndof + s] = 0.0;
    return SPRING_OK;
}

int spring_path_qpoints(spring_ctx* c, int n_nodes, const double* q_high_sym, int* n_rows, double* qpoints,
                        double* dist, int* zero_centered) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->crystal_set, "crystal"));
    if (n_nodes < 1 || !q_high_sym || !n_rows) return fail(c, SPRING_ERR_ARG, "n_nodes < 1 or NULL q_high_sym / n_rows");
    for (int k = 0; k < n_nodes; ++k)
        if (!(q_high_sym[4 * k + 3] >= 0.0)) return fail(c, SPRING_ERR_ARG, "negative point count at node %d", k + 1);
    *n_rows = path_points(c->G, n_nodes, q_high_sym, qpoints, dist, zero_centered);
    return SPRING_OK;
}

int spring_linewidth_path(spring_ctx* c, int n_q0, const double* q0, const int* zero_centered, int delta_mode,
                          double sigma, double* lw, double* omega_q0) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->fc2_set, "FC2"));
    SPRING_CHECK(need(c, c->fc3_set, "FC3"));
    SPRING_CHECK(need(c, c->mesh_set, "mesh"));
    SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    if (!c->mesh_zc) return fail(c, SPRING_ERR_STATE, "the path mode needs the zero-centred mesh (spring_make_mesh zero_centered = 1)");
    if (n_q0 < 0 || (n_q0 > 0 && (!q0 || !zero_centered))) return fail(c, SPRING_ERR_ARG, "n_q0 < 0 or NULL q0 / flags");
    if (delta_mode != SPRING_DELTA_GAUSS && delta_mode != SPRING_DELTA_TETRA)
        return fail(c, SPRING_ERR_ARG, "delta_mode must be SPRING_DELTA_GAUSS or SPRING_DELTA_TETRA");
    if (delta_mode == SPRING_DELTA_GAUSS && !(sigma > 0.0)) return fail(c, SPRING_ERR_ARG, "sigma must be > 0");
    if (c->nT > 9) return fail(c, SPRING_ERR_UNSUPPORTED, "the path mode handles at most 9 temperatures per call");
    if (n_q0 == 0) return SPRING_OK;
    std::vector<double> buf(lw ? (size_t)c->nT * n_q0 * c->ndof : 0);
    SPRING_CHECK(run_path(c, n_q0, q0, zero_centered, delta_mode, sigma, lw ? buf.data() : nullptr, omega_q0));
    if (lw) std::memcpy(lw, buf.data(), sizeof(double) * buf.size());  // [T][p][s] is lw(Ndof, n_q0, n_temps)
    return SPRING_OK;
}

int spring_mlp_init(spring_ctx* c, unsigned long long seed) {
    CTX_ENTER(c);
    if (mlp_num_params() != SPRING_MLP_PARAMS) return fail(c, SPRING_ERR_STATE, "network size mismatch");
    return run_mlp_init(c, seed);
}

int spring_mlp_set_params(spring_ctx* c, const float* params) {
    CTX_ENTER(c);
    if (!params) return fail(c, SPRING_ERR_ARG, "params is NULL");
    return run_mlp_set(c, params);
}

int spring_mlp_get_params(spring_ctx* c, float* params) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->mlp.set, "network parameters"));
    if (!params) return fail(c, SPRING_ERR_ARG, "params is NULL");
    return d2h(c, params, c->mlp.p.p, sizeof(float) * SPRING_MLP_PARAMS, "network parameters");
}

int spring_mlp_loss_grad(spring_ctx* c, int n, const float* X, const float* y, float* loss, float* grad) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->mlp.set, "network parameters"));
    if (n < 1 || !X || !y) return fail(c, SPRING_ERR_ARG, "n < 1 or NULL X / y");
    return run_mlp_loss_grad(c, n, X, y, loss, grad);
}

int spring_mlp_train(spring_ctx* c, int n, const float* X, const float* y, int epochs, int batch, float lr,
                     unsigned long long seed, float* epoch_loss) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->mlp.set, "network parameters"));
    if (n < 1 || !X || !y || epochs < 0 || batch < 1 || !(lr > 0.0f))
        return fail(c, SPRING_ERR_ARG, "n, batch >= 1, epochs >= 0, lr > 0 and non-NULL X / y are required");
    return run_mlp_train(c, n, X, y, epochs, batch, lr, seed, epoch_loss);
}

int spring_mlp_predict(spring_ctx* c, int n, const float* X, float* y, int bf16) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->mlp.set, "network parameters"));
    if (n < 0 || (n > 0 && (!X || !y))) return fail(c, SPRING_ERR_ARG, "n < 0 or NULL X / y");
    if (n == 0) return SPRING_OK;
    return run_mlp_predict(c, n, X, y, bf16);
}

int spring_set_precision(spring_ctx* c, int precision) {
    CTX_ENTER(c);
    if (precision != SPRING_FP64 && precision != SPRING_BF16 && precision != SPRING_BF16X3)
        return fail(c, SPRING_ERR_ARG, "precision must be SPRING_FP64, SPRING_BF16 or SPRING_BF16X3");
    c->precision = precision;
    return SPRING_OK;
}

int spring_reset_linewidths(spring_ctx* c) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    return zero(c, c->d_lw_all.p, sizeof(double) * c->nT * c->nq0 * c->ndof, "LW_Allq0");
}

int spring_get_linewidths(spring_ctx* c, double* out) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    if (!out) return fail(c, SPRING_ERR_ARG, "output is NULL");
    return d2h(c, out, c->d_lw_all.p, sizeof(double) * c->nT * c->nq0 * c->ndof, "LW_Allq0");
}

int spring_set_linewidths(spring_ctx* c, const double* in) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    if (!in) return fail(c, SPRING_ERR_ARG, "input is NULL");
    SPRING_CHECK(h2d(c, c->d_lw_all.p, in, sizeof(double) * c->nT * c->nq0 * c->ndof, "LW_Allq0"));
    return spring_synchronize(c);
}

int spring_kappa_rta(spring_ctx* c, int symm, int nsym, const double* rxyz, const int* s_range, double* kappa,
                     double* mode_k) {
    CTX_ENTER(c);
    SPRING_CHECK(need(c, c->irr_set, "irreducible q-points"));
    SPRING_CHECK(need(c, c->ph_irr.set, "irreducible-point phonons"));
    if (!symm) SPRING_CHECK(need(c, c->ph_grid.set, "grid phonons"));
    if (symm && (nsym < 1 || !rxyz)) return fail(c, SPRING_ERR_ARG, "symmetrised kappa needs Rxyz");
    int lo = 1, hi = c->ndof;
    if (s_range) { lo = s_range[0]; hi = s_range[1]; }
    if (lo < 1 || hi > c->ndof || lo > hi) return fail(c, SPRING_ERR_ARG, "s_range out of range");
    SPRING_CHECK(dalloc(c, c->d_kappa, (size_t)c->nT * 9 * (1 + c->ndof), "kappa"));
    if (symm) {
        SPRING_CHECK(dalloc(c, c->d_rxyz, (size_t)nsym * 9, "Rxyz"));
        SPRING_CHECK(h2d(c, c->d_rxyz.p, rxyz, sizeof(double) * 9 * nsym, "Rxyz"));
    }
    double* dk = c->d_kappa.p;
    double* dm = c->d_kappa.p + (size_t)c->nT * 9;
    SPRING_CHECK(run_kappa_rta(c, symm, nsym, c->d_rxyz.p, lo - 1, hi - 1, dk, dm));
    if (kappa) SPRING_CHECK(d2h(c, kappa, dk, sizeof(double) * 9 * c->nT, "kappa"));
    if (mode_k) SPRING_CHECK(d2h(c, mode_k, dm, sizeof(double) * 9 * c->ndof * c->nT, "mode kappa"));
    return SPRING_OK;
}

}  // extern "C"

namespace spring {

// The checks and prerequisites of a Gaussian three-phonon linewidth request, as spring_linewidth3
// makes them (used by the batch entry points).
int prepare_lw3(spring_ctx* c, int i0_first, int n_q0, const int* pol3, Pol* pol) {
    SPRING_CHECK(check_q0_range(c, i0_first, n_q0));
    SPRING_CHECK(ready3(c));
    SPRING_CHECK(check_pol(c, pol3));
    SPRING_CHECK(ensure_enum3(c));
    SPRING_CHECK(pairoff_host(c, c->ps_irr));  // the batch kernel's descriptors take host pair ranges
    *pol = make_pol(c, pol3);
    return SPRING_OK;
}

int lw_out(spring_ctx* c, const double* d_src, int q0_first, int n_q0, double* out) {
    return copy_lw_out(c, d_src, q0_first, n_q0, out);
}

}  // namespace spring
