// Batched three-phonon linewidths: several workloads (cells, meshes,
// temperature sets) in one persistent launch.
//
// Each request is spring_linewidth3 with the Gaussian delta on its context
// (q0 loop body of src/Kappa/Src/main.f90:552-715, ScatterMatEl /
// ScatterProbability + CalculateLinewidth, ThirdOrder_m.f90:278-543).  The
// requests' (pair, s0-block) work items are concatenated, heaviest workload
// first, and one persistent CTA per slot takes items from a global counter
// (`chunk` at a time), so uneven workloads (Ndof 6 and 24, 12^3 to 20^3 meshes,
// 1 to 9 temperatures) share one launch without tail effects.  Each item runs
// the any-cell FP64 V3 work item of k_v3.cu against its workload's
// descriptor (staged in shared memory when the workload changes).  The zero
// fills, the kernel and the LW_Allq0 updates are captured in one CUDA graph.
//
// Autotuner: threads per CTA, CTAs per SM, the s0 block of large cells and the
// items per scheduler step are chosen by timing the batch itself (CUDA events),
// coordinate by coordinate; the choice is cached for the process by the batch
// shape.
// Roofline: FP64 FMA, as k_v3 (41.3 kflop per pair for Ndof 6; 8.0 Mflop for
// Ndof 24).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "v3item.cuh"
#include "v3sitem.cuh"

namespace spring {
namespace {

constexpr int BT = s3::THREADS;  // threads per CTA: the two-atom group layout needs exactly 288

struct BatchDesc {
    int kind;        // 0: two-atom groups of s3::PP pairs (k_v3s layout), 1: any cell, (pair, s0 block)
    V3Args a;        // kind 1 (and the fold's sizes for both kinds)
    V3Ptrs P;        // kind 1 (out_lw also read by the fold)
    s3::S3Args a3;   // kind 0
    s3::S3Ptrs P3;   // kind 0
    double* lw_all;  // LW_Allq0 of the context
    long long fold0, fold_n;  // this request's slab [T][q0 range][s] in the fold kernel's index space
};

__global__ void __launch_bounds__(BT, 2) k_v3_batch(const BatchDesc* __restrict__ desc, const long long* __restrict__ off,
                                                    int nw, int chunk, unsigned long long* __restrict__ ctr) {
    extern __shared__ __align__(16) double2 smem2[];
    s3::Smem& S = *reinterpret_cast<s3::Smem*>(smem2);
    __shared__ long long s_it;
    __shared__ int s_w, s_new;
    __shared__ BatchDesc s_d;
    if (threadIdx.x == 0) s_w = -1;
    const long long total = off[nw];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_it = (long long)atomicAdd(ctr, (unsigned long long)chunk);
        __syncthreads();
        const long long it0 = s_it;
        if (it0 >= total) break;
        const long long it1 = min(it0 + (long long)chunk, total);
        for (long long it = it0; it < it1; ++it) {
            int w = 0;
            while (w + 1 < nw && off[w + 1] <= it) ++w;
            __syncthreads();
            if (threadIdx.x == 0) {
                s_new = w != s_w;
                if (s_new) {
                    s_d = desc[w];
                    s_w = w;
                }
            }
            __syncthreads();
            const long long local = it - off[w];
            if (s_d.kind == 0) {
                if (s_new) s3::v3s_stage(S, s_d.P3);  // v3s_group syncs before reading the constants
                s3::v3s_group<0>(S, s_d.a3, s_d.P3, (int)local);
            } else {
                const int pr = s_d.a.pair_first + (int)(local / s_d.a.nsb);
                const int s0b = (int)(local % s_d.a.nsb) * s_d.a.sb;
                v3_item<0>(s_d.a, s_d.P, pr, s0b, smem2);
            }
        }
    }
}

// LW_Allq0 += lw for every request's q0 range (weight 1, main.f90:584).
__global__ void k_batch_fold(const BatchDesc* __restrict__ desc, int nw, long long total) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        int w = 0;
        while (w + 1 < nw && desc[w + 1].fold0 <= i) ++w;
        const BatchDesc& d = desc[w];
        const long long k = i - d.fold0;
        const int n = d.a.n;
        const long long per_t = d.fold_n / d.a.nT;  // n_q0 * n
        const int t = (int)(k / per_t);
        const long long r = k % per_t;
        const size_t idx = ((size_t)t * d.a.nq0 + d.a.q0_first) * n + r;
        d.lw_all[idx] += d.P.out_lw[idx];
    }
}

struct Guard {
    int prev = -1;
    explicit Guard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Guard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

std::map<std::string, std::vector<int>>& tune_cache() {
    static std::map<std::string, std::vector<int>> m;
    return m;
}

}  // namespace
}  // namespace spring

using spring::BatchDesc;

struct spring_batch {
    struct Work {
        spring_ctx* c;
        int q0, n_q0;
        double sigma;
        spring::Pol pol;
        long long pairs = 0, items = 0;
        int kind = 1;       // 0: two-atom groups, 1: any cell, 2: tensor-core pass (outside the kernel)
        double cost = 0.0;  // per item, for the heaviest-first order
    };
    std::vector<Work> work;
    // Gaussian linewidths at path points of a context (LineWidth.x path mode), queued in the graph
    // after the persistent kernel; the plan holds every buffer, allocated at the first run.
    struct PathReq {
        spring_ctx* c;
        int n_path;
        std::vector<double> q;
        std::vector<int> zc;
        double sigma;
        spring::PathPlan plan;
        bool ready = false;
    };
    std::vector<PathReq> paths;
    std::string err;
    // two-atom group path (1: where the cell fits), CTAs per SM (0: occupancy limit), s0 block for
    // Ndof > 12 (0: 6), work items per scheduler step
    int cfg[4] = {1, 0, 0, 1};
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_sync = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> graph_key;  // launch shape the graph was captured for
    BatchDesc* d_desc = nullptr;
    long long* d_off = nullptr;
    unsigned long long* d_ctr = nullptr;
    int nw_alloc = 0;
    double last_ms = 0.0;
};

namespace {

int bfail(spring_batch* b, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    b->err = buf;
    return code;
}

int bcuda(spring_batch* b, cudaError_t e, const char* what) {
    return e == cudaSuccess ? SPRING_OK : bfail(b, SPRING_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define BCHECK(expr)                      \
    do {                                  \
        const int _rc = (expr);           \
        if (_rc != SPRING_OK) return _rc; \
    } while (0)

void drop_graph(spring_batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_key.clear();
}

std::string shape_key(const spring_batch* b) {
    std::string k;
    char buf[160];
    for (const auto& w : b->work) {
        snprintf(buf, sizeof buf, "%d:%d:%d:%d:%lld;", w.c->ndof, w.c->nq, w.c->nT, w.c->na3, w.pairs);
        k += buf;
    }
    return k;
}

// Requests that the tensor-core pass takes (two-atom cells with at most 8-atom FC3 clusters on a
// context set to BF16 or BF16x3, as in spring_linewidth3): they run through it, not as items of the
// persistent FP64 kernel.
bool tc_request(const spring_ctx* c) { return c->precision != SPRING_FP64 && c->nb == 2 && c->na3 <= 8; }

// Device descriptors of every request for the configuration in b->cfg, in heaviest-first order;
// returns the shared-memory size, the item offsets and the fold total on the host too.
int build_desc(spring_batch* b, std::vector<BatchDesc>& D, std::vector<long long>& off, size_t* smem,
               long long* fold_total) {
    const int nw = (int)b->work.size();
    std::vector<int> order(nw);
    for (int i = 0; i < nw; ++i) order[i] = i;
    const int sb_big = b->cfg[2] > 0 ? b->cfg[2] : 6;
    for (auto& w : b->work) {
        spring_ctx* c = w.c;
        const int n = c->ndof, sb = n <= 12 ? n : sb_big;
        const spring::PairSet& ps = c->ps_irr;
        if (spring::pairoff_host(c, ps) != SPRING_OK) return bfail(b, SPRING_ERR_CUDA, "%s", c->err.c_str());
        w.pairs = ps.h_pairoff[w.q0 + w.n_q0] - ps.h_pairoff[w.q0];
        w.kind = (b->cfg[0] && c->nb == spring::s3::NB && c->na3 == spring::s3::NA && c->nT <= spring::s3::MAXT) ? 0 : 1;
        if (tc_request(c)) w.kind = 2;
        if (w.kind == 2) {
            w.items = 0;  // the tensor-core pass runs it, beside the persistent kernel
            w.cost = 0.0;
        } else if (w.kind == 0) {
            w.items = (w.pairs + spring::s3::PP - 1) / spring::s3::PP;
            w.cost = spring::s3::PP * (27.0 * 4 * c->na3 * c->na3 + 8.0 * n * n * n * n);
        } else {
            w.items = w.pairs * ((n + sb - 1) / sb);
            w.cost = (double)n * n * n * sb + 27.0 * c->na3 * c->na3 * n * n;
        }
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->work[x].cost > b->work[y].cost; });
    D.assign(nw, BatchDesc{});
    off.assign(nw + 1, 0);
    *smem = 0;
    long long fold = 0;
    for (int k = 0; k < nw; ++k) {
        const auto& w = b->work[order[k]];
        spring_ctx* c = w.c;
        const int n = c->ndof, sb = n <= 12 ? n : sb_big;
        spring::V3Args& a = D[k].a;
        a.nb = c->nb;
        a.n = n;
        a.na = c->na3;
        a.nq = c->nq;
        a.nq0 = c->ps_irr.n0;
        a.nT = c->nT;
        a.q0_first = w.q0;
        a.sb = sb;
        a.nsb = (n + sb - 1) / sb;
        a.mfac = spring::host_constants().Sctr3THz2 / double(c->nq);
        a.pair_first = c->ps_irr.h_pairoff[w.q0];
        a.onebysigma = 1.0 / w.sigma;
        a.onebysigma2 = a.onebysigma * a.onebysigma;
        for (int i = 0; i < 3; ++i) {
            a.pol_lo[i] = w.pol.lo[i];
            a.pol_hi[i] = w.pol.hi[i];
        }
        const spring::Q0View v = spring::irr_view(c);
        D[k].P = spring::V3Ptrs{c->ps_irr.pairs.p, c->ps_irr.pair_q0.p, c->d_fc3.p, c->d_fc3_posr.p,
                                c->d_fc3_btyp.p, c->d_mass_rs.p, c->d_qpnt.p, v.q0_int, v.q0_grid, v.evec, v.omega,
                                v.oneby, c->ph_grid.evec.p, c->ph_grid.omega.p, c->ph_grid.oneby.p,
                                c->ph_grid.nbe.p, c->d_lw_tmp.p, c->d_p3.p, nullptr};
        D[k].kind = w.kind;
        if (w.kind == 0) {
            spring::s3::S3Args& a3 = D[k].a3;
            a3.nq = c->nq;
            a3.nT = c->nT;
            a3.nq0 = c->ps_irr.n0;
            a3.q0_first = w.q0;
            a3.pair_first = c->ps_irr.h_pairoff[w.q0];
            a3.pair_end = c->ps_irr.h_pairoff[w.q0 + w.n_q0];
            a3.plist = nullptr;
            a3.ngroups = (int)w.items;
            a3.mfac = a.mfac;
            a3.onebysigma = a.onebysigma;
            a3.onebysigma2 = a.onebysigma2;
            for (int i = 0; i < 3; ++i) {
                a3.pol_lo[i] = w.pol.lo[i];
                a3.pol_hi[i] = w.pol.hi[i];
            }
            D[k].P3 = spring::s3::S3Ptrs{c->ps_irr.pairs.p, c->ps_irr.pair_q0.p, c->d_fc3.p, c->d_fc3_posr.p,
                                 c->d_fc3_btyp.p, c->d_fc3_off.p, c->d_mass_rs.p, c->d_qpnt.p, v.q0_int, v.q0_grid,
                                 v.evec, v.omega, v.oneby, c->ph_grid.evec.p, c->ph_grid.omega.p,
                                 c->ph_grid.oneby.p, c->ph_grid.nbe.p, c->d_lw_tmp.p, c->d_p3.p, nullptr};
            *smem = std::max(*smem, sizeof(spring::s3::Smem));
        } else {
            *smem = std::max(*smem, spring::v3_smem(n, c->na3, sb, c->nT));
        }
        D[k].lw_all = c->d_lw_all.p;
        D[k].fold0 = fold;
        D[k].fold_n = w.kind == 2 ? 0 : (long long)c->nT * w.n_q0 * n;  // kind 2 folds after its own pass
        fold += D[k].fold_n;
        off[k + 1] = off[k] + w.items;
    }
    *fold_total = fold;
    return SPRING_OK;
}

// Per-request prerequisites (pair lists, scratch) on each context; idempotent.
int prepare(spring_batch* b) {
    if (b->work.empty()) return bfail(b, SPRING_ERR_STATE, "the batch holds no requests");
    for (auto& w : b->work) {
        spring_ctx* c = w.c;
        spring::Pol pol;
        const int rc = spring::prepare_lw3(c, w.q0 + 1, w.n_q0, nullptr, &pol);
        if (rc != SPRING_OK) return bfail(b, rc, "request on a context: %s", c->err.c_str());
        const size_t nl = (size_t)c->nT * c->nq0 * c->ndof;
        if (spring::dalloc(c, c->d_lw_tmp, nl, "linewidth scratch") != SPRING_OK ||
            spring::dalloc(c, c->d_p3, (size_t)c->nq0 * c->ndof, "phase-space scratch") != SPRING_OK)
            return bfail(b, SPRING_ERR_ALLOC, "%s", c->err.c_str());
    }
    return SPRING_OK;
}

// Zero the scratch of every context, run the persistent kernel and (fold) the LW_Allq0 updates on
// b->stream.
int enqueue(spring_batch* b, const std::vector<BatchDesc>& D, const std::vector<long long>& off, size_t smem,
            long long fold_total, bool fold) {
    const int nw = (int)D.size();
    std::vector<spring_ctx*> seen;
    for (const auto& w : b->work) {
        spring_ctx* c = w.c;
        if (std::find(seen.begin(), seen.end(), c) != seen.end()) continue;
        seen.push_back(c);
        BCHECK(bcuda(b, cudaMemsetAsync(c->d_lw_tmp.p, 0, sizeof(double) * c->nT * c->nq0 * c->ndof, b->stream),
                     "batch scratch"));
        BCHECK(bcuda(b, cudaMemsetAsync(c->d_p3.p, 0, sizeof(double) * c->nq0 * c->ndof, b->stream), "batch scratch"));
    }
    BCHECK(bcuda(b, cudaMemsetAsync(b->d_ctr, 0, sizeof(unsigned long long), b->stream), "batch counter"));
    const int threads = spring::BT;
    int occ = 0;
    BCHECK(bcuda(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, spring::k_v3_batch, threads, smem),
                 "batch occupancy"));
    if (occ < 1) return bfail(b, SPRING_ERR_UNSUPPORTED, "batch kernel does not fit an SM (%zu bytes)", smem);
    const int per_sm = b->cfg[1] > 0 ? std::min(b->cfg[1], occ) : occ;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    const long long total = off[nw];
    const int grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, total));
    spring::k_v3_batch<<<grid, threads, smem, b->stream>>>(b->d_desc, b->d_off, nw, std::max(1, b->cfg[3]), b->d_ctr);
    BCHECK(bcuda(b, cudaGetLastError(), "k_v3_batch"));
    if (fold && fold_total > 0) {
        const int fb = (int)std::min<long long>((fold_total + 255) / 256, (long long)sms * 8);
        spring::k_batch_fold<<<fb, 256, 0, b->stream>>>(b->d_desc, nw, fold_total);
        BCHECK(bcuda(b, cudaGetLastError(), "k_batch_fold"));
    }
    return SPRING_OK;
}

int upload(spring_batch* b, const std::vector<BatchDesc>& D, const std::vector<long long>& off, size_t smem) {
    const int nw = (int)D.size();
    if (nw > b->nw_alloc) {
        if (b->d_desc) cudaFree(b->d_desc);
        if (b->d_off) cudaFree(b->d_off);
        b->d_desc = nullptr;
        b->d_off = nullptr;
        BCHECK(bcuda(b, cudaMalloc(&b->d_desc, sizeof(BatchDesc) * nw), "batch descriptors"));
        BCHECK(bcuda(b, cudaMalloc(&b->d_off, sizeof(long long) * (nw + 1)), "batch offsets"));
        b->nw_alloc = nw;
    }
    if (!b->d_ctr) BCHECK(bcuda(b, cudaMalloc(&b->d_ctr, sizeof(unsigned long long)), "batch counter"));
    if (smem > 227 * 1024) return bfail(b, SPRING_ERR_UNSUPPORTED, "batch work item needs %zu bytes of shared memory", smem);
    BCHECK(bcuda(b, cudaFuncSetAttribute(spring::k_v3_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                 "batch shared memory"));
    BCHECK(bcuda(b, cudaMemcpyAsync(b->d_desc, D.data(), sizeof(BatchDesc) * nw, cudaMemcpyHostToDevice, b->stream),
                 "batch descriptors"));
    BCHECK(bcuda(b, cudaMemcpyAsync(b->d_off, off.data(), sizeof(long long) * (nw + 1), cudaMemcpyHostToDevice,
                                    b->stream),
                 "batch offsets"));
    return bcuda(b, cudaStreamSynchronize(b->stream), "batch descriptors");
}

// Order the batch stream after the contexts' streams (and, at the end, the contexts after it).
int join_ctx_in(spring_batch* b, spring_ctx* c) {
    if (c->stream == b->stream) return SPRING_OK;
    BCHECK(bcuda(b, cudaEventRecord(b->ev_sync, c->stream), "batch join"));
    return bcuda(b, cudaStreamWaitEvent(b->stream, b->ev_sync, 0), "batch join");
}
int join_ctx_out(spring_batch* b, spring_ctx* c) {
    if (c->stream == b->stream) return SPRING_OK;
    BCHECK(bcuda(b, cudaEventRecord(b->ev_sync, b->stream), "batch join"));
    return bcuda(b, cudaStreamWaitEvent(c->stream, b->ev_sync, 0), "batch join");
}
int join_in(spring_batch* b) {
    for (const auto& w : b->work) BCHECK(join_ctx_in(b, w.c));
    for (const auto& p : b->paths) BCHECK(join_ctx_in(b, p.c));
    return SPRING_OK;
}
int join_out(spring_batch* b) {
    for (const auto& w : b->work) BCHECK(join_ctx_out(b, w.c));
    for (const auto& p : b->paths) BCHECK(join_ctx_out(b, p.c));
    return SPRING_OK;
}

// Buffers of every path request (once) and the upload of its points.
int prepare_paths(spring_batch* b) {
    for (auto& p : b->paths) {
        if (p.ready) continue;
        spring::Guard g(p.c->device);
        const int rc = spring::path_prepare(p.c, p.plan, p.n_path, p.q.data(), p.zc.data());
        if (rc != SPRING_OK) return bfail(b, rc, "path request: %s", p.c->err.c_str());
        p.ready = true;
    }
    return SPRING_OK;
}

// The launches of every path request on the batch stream (captured into the graph).
int enqueue_paths(spring_batch* b) {
    for (auto& p : b->paths) {
        spring_ctx* c = p.c;
        cudaStream_t own = c->stream;
        const bool prof = c->profiling;
        c->stream = b->stream;
        c->profiling = false;  // no per-launch timing events inside the graph
        const int rc = spring::path_enqueue(c, p.plan, SPRING_DELTA_GAUSS, p.sigma);
        c->stream = own;
        c->profiling = prof;
        if (rc != SPRING_OK) return bfail(b, rc, "path request: %s", c->err.c_str());
    }
    return SPRING_OK;
}

// The tensor-core requests after the graph (which zeroed their scratch): the pass of
// spring_linewidth3 on each context's stream, then its LW_Allq0 update; the batch stream waits for
// them.
int run_tc_requests(spring_batch* b) {
    for (const auto& w : b->work) {
        if (w.kind != 2) continue;
        spring_ctx* c = w.c;
        BCHECK(join_ctx_out(b, c));
        int rc = spring::run_v3_gauss(c, w.q0, w.n_q0, w.sigma, w.pol, c->d_lw_tmp.p, c->d_p3.p);
        if (rc == SPRING_OK) rc = spring::run_axpy_lw(c, 1.0, c->d_lw_tmp.p, c->d_lw_all.p, w.q0, w.n_q0);
        if (rc != SPRING_OK) return bfail(b, rc, "tensor-core request: %s", c->err.c_str());
        BCHECK(join_ctx_in(b, c));
    }
    return SPRING_OK;
}

// One timed run without the LW_Allq0 update (for the tuner).
int timed_trial(spring_batch* b, double* ms) {
    std::vector<BatchDesc> D;
    std::vector<long long> off;
    size_t smem = 0;
    long long fold_total = 0;
    BCHECK(build_desc(b, D, off, &smem, &fold_total));
    BCHECK(upload(b, D, off, smem));
    BCHECK(bcuda(b, cudaEventRecord(b->ev0, b->stream), "batch timing"));
    BCHECK(enqueue(b, D, off, smem, fold_total, false));
    BCHECK(bcuda(b, cudaEventRecord(b->ev1, b->stream), "batch timing"));
    BCHECK(bcuda(b, cudaEventSynchronize(b->ev1), "batch timing"));
    float t = 0.0f;
    BCHECK(bcuda(b, cudaEventElapsedTime(&t, b->ev0, b->ev1), "batch timing"));
    *ms = t;
    return SPRING_OK;
}

}  // namespace

extern "C" {

int spring_batch_create(spring_batch** out) {
    if (!out) return SPRING_ERR_ARG;
    *out = new spring_batch();
    return SPRING_OK;
}

int spring_batch_destroy(spring_batch* b) {
    if (!b) return SPRING_OK;
    if (b->device >= 0) {
        spring::Guard g(b->device);
        if (b->stream) cudaStreamSynchronize(b->stream);
        drop_graph(b);
        if (b->d_desc) cudaFree(b->d_desc);
        if (b->d_off) cudaFree(b->d_off);
        if (b->d_ctr) cudaFree(b->d_ctr);
        if (b->ev0) cudaEventDestroy(b->ev0);
        if (b->ev1) cudaEventDestroy(b->ev1);
        if (b->ev_sync) cudaEventDestroy(b->ev_sync);
        for (auto& p : b->paths) spring::path_release(p.plan);
    }
    delete b;
    return SPRING_OK;
}

const char* spring_batch_last_error(const spring_batch* b) { return b ? b->err.c_str() : "batch is NULL"; }

int spring_batch_add_linewidth3(spring_batch* b, spring_ctx* c, int i0_first, int n_q0, double sigma, const int* pol3,
                                int* index) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (!c) return bfail(b, SPRING_ERR_ARG, "context is NULL");
    if (b->device >= 0 && c->device != b->device)
        return bfail(b, SPRING_ERR_ARG, "context on device %d, batch on device %d", c->device, b->device);
    if (!(sigma > 0.0)) return bfail(b, SPRING_ERR_ARG, "sigma must be > 0");
    spring::Guard g(c->device);
    spring::Pol pol;
    const int rc = spring::prepare_lw3(c, i0_first, n_q0, pol3, &pol);
    if (rc != SPRING_OK) return bfail(b, rc, "%s", c->err.c_str());
    if (n_q0 == 0) return bfail(b, SPRING_ERR_ARG, "empty q0 range");
    for (const auto& w : b->work)
        if (w.c == c && i0_first - 1 < w.q0 + w.n_q0 && w.q0 < i0_first - 1 + n_q0)
            return bfail(b, SPRING_ERR_ARG, "q0 range overlaps an earlier request on the same context");
    if (b->device < 0) {
        b->device = c->device;
        b->stream = c->stream;
        if (cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_sync, cudaEventDisableTiming) != cudaSuccess)
            return bfail(b, SPRING_ERR_CUDA, "batch events");
    }
    spring_batch::Work w;
    w.c = c;
    w.q0 = i0_first - 1;
    w.n_q0 = n_q0;
    w.sigma = sigma;
    w.pol = pol;
    b->work.push_back(w);
    drop_graph(b);
    if (index) *index = (int)b->work.size() - 1;
    return SPRING_OK;
}

int spring_batch_add_path(spring_batch* b, spring_ctx* c, int n_path, const double* q_path, const int* zero_centered,
                          double sigma, int* index) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (!c) return bfail(b, SPRING_ERR_ARG, "context is NULL");
    if (b->device < 0) return bfail(b, SPRING_ERR_STATE, "add a linewidth request first (it binds the batch's device)");
    if (c->device != b->device)
        return bfail(b, SPRING_ERR_ARG, "context on device %d, batch on device %d", c->device, b->device);
    if (n_path < 1 || !q_path || !zero_centered) return bfail(b, SPRING_ERR_ARG, "n_path < 1 or NULL points / flags");
    if (!(sigma > 0.0)) return bfail(b, SPRING_ERR_ARG, "sigma must be > 0");
    if (!c->fc2_set || !c->fc3_set || !c->mesh_set || !c->ph_grid.set)
        return bfail(b, SPRING_ERR_STATE, "the context needs FC2, FC3, the mesh and the grid phonons");
    if (!c->mesh_zc) return bfail(b, SPRING_ERR_STATE, "the path mode needs the zero-centred mesh");
    if (c->nT > 9) return bfail(b, SPRING_ERR_UNSUPPORTED, "the path mode handles at most 9 temperatures");
    spring_batch::PathReq r;
    r.c = c;
    r.n_path = n_path;
    r.q.assign(q_path, q_path + 3 * (size_t)n_path);
    r.zc.assign(zero_centered, zero_centered + n_path);
    r.sigma = sigma;
    b->paths.push_back(std::move(r));
    drop_graph(b);
    if (index) *index = (int)b->paths.size() - 1;
    return SPRING_OK;
}

int spring_batch_path_result(spring_batch* b, int index, double* lw, double* omega) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (index < 0 || index >= (int)b->paths.size()) return bfail(b, SPRING_ERR_ARG, "no path request %d", index);
    auto& p = b->paths[index];
    if (!p.ready || !b->exec) return bfail(b, SPRING_ERR_STATE, "the batch has not run");
    spring::Guard g(b->device);
    BCHECK(join_ctx_out(b, p.c));  // the context's stream follows the batch's last run
    const int rc = spring::path_fetch(p.c, p.plan, lw, omega);
    return rc == SPRING_OK ? SPRING_OK : bfail(b, rc, "%s", p.c->err.c_str());
}

int spring_batch_set_config(spring_batch* b, const int* config) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (!config) return bfail(b, SPRING_ERR_ARG, "config is NULL");
    if (config[0] != 0 && config[0] != 1) return bfail(b, SPRING_ERR_ARG, "two-atom path must be 0 or 1");
    if (config[1] < 0 || config[1] > 16) return bfail(b, SPRING_ERR_ARG, "CTAs per SM must be in [0, 16]");
    if (config[2] != 0 && config[2] != 6 && config[2] != 12 && config[2] != 24)
        return bfail(b, SPRING_ERR_ARG, "s0 block must be 0, 6, 12 or 24");
    if (config[3] < 1 || config[3] > 64) return bfail(b, SPRING_ERR_ARG, "items per step must be in [1, 64]");
    for (int i = 0; i < 4; ++i) b->cfg[i] = config[i];
    drop_graph(b);
    return SPRING_OK;
}

int spring_batch_get_config(const spring_batch* b, int* config) {
    if (!b || !config) return SPRING_ERR_ARG;
    for (int i = 0; i < 4; ++i) config[i] = b->cfg[i];
    return SPRING_OK;
}

int spring_batch_tune(spring_batch* b, int* config, double* best_ms, int* n_tried) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (b->work.empty()) return bfail(b, SPRING_ERR_STATE, "the batch holds no requests");
    spring::Guard g(b->device);
    BCHECK(prepare(b));
    BCHECK(join_in(b));
    bool big = false;
    for (const auto& w : b->work) big = big || w.c->ndof > 12;
    int best[4] = {1, 0, big ? 6 : 0, 1};
    double bms = 0.0;
    int tried = 0;
    auto trial = [&](const int* cand, double* ms) {
        for (int i = 0; i < 4; ++i) b->cfg[i] = cand[i];
        ++tried;
        return timed_trial(b, ms);
    };
    BCHECK(trial(best, &bms));  // warm-up of the baseline
    BCHECK(trial(best, &bms));
    auto sweep = [&](int k, const std::vector<int>& vals) -> int {
        for (int v : vals) {
            if (v == best[k]) continue;
            int cand[4] = {best[0], best[1], best[2], best[3]};
            cand[k] = v;
            double ms = 0.0;
            const int rc = trial(cand, &ms);
            if (rc == SPRING_ERR_UNSUPPORTED) {  // does not fit (shared memory): not a candidate
                b->err.clear();
                continue;
            }
            BCHECK(rc);
            if (ms < bms) {
                bms = ms;
                best[k] = v;
            }
        }
        return SPRING_OK;
    };
    BCHECK(sweep(0, {0, 1}));
    BCHECK(sweep(1, {1, 2, 3, 4}));
    if (big) BCHECK(sweep(2, {6, 12, 24}));
    BCHECK(sweep(3, {1, 4, 16}));
    for (int i = 0; i < 4; ++i) b->cfg[i] = best[i];
    spring::tune_cache()[shape_key(b)] = std::vector<int>(best, best + 4);
    drop_graph(b);
    BCHECK(join_out(b));
    if (config)
        for (int i = 0; i < 4; ++i) config[i] = best[i];
    if (best_ms) *best_ms = bms;
    if (n_tried) *n_tried = tried;
    return SPRING_OK;
}

int spring_batch_run(spring_batch* b) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (b->work.empty()) return bfail(b, SPRING_ERR_STATE, "the batch holds no requests");
    spring::Guard g(b->device);
    BCHECK(prepare(b));
    BCHECK(prepare_paths(b));
    // a tuned configuration of the same shape, if this batch has not been configured otherwise
    if (b->cfg[0] == 1 && b->cfg[1] == 0 && b->cfg[2] == 0 && b->cfg[3] == 1) {
        std::vector<BatchDesc> D0;
        std::vector<long long> o0;
        size_t s0 = 0;
        long long f0 = 0;
        BCHECK(build_desc(b, D0, o0, &s0, &f0));  // fills the item counts of the shape key
        auto it = spring::tune_cache().find(shape_key(b));
        if (it != spring::tune_cache().end())
            for (int i = 0; i < 4; ++i) b->cfg[i] = it->second[i];
    }
    // Descriptors are rebuilt and uploaded every run (the graph reads them from device memory), so
    // new phonons or reallocated buffers are picked up; the graph is captured again only when its
    // launch shape (configuration, work split, shared memory, descriptor buffer) changes.
    std::vector<BatchDesc> D;
    std::vector<long long> off;
    size_t smem = 0;
    long long fold_total = 0;
    BCHECK(build_desc(b, D, off, &smem, &fold_total));
    BCHECK(join_in(b));
    BCHECK(upload(b, D, off, smem));
    std::vector<long long> key(b->cfg, b->cfg + 4);
    key.push_back((long long)smem);
    key.push_back(fold_total);
    key.push_back((long long)reinterpret_cast<uintptr_t>(b->d_desc));
    key.insert(key.end(), off.begin(), off.end());
    for (const auto& p : b->paths) key.push_back((long long)reinterpret_cast<uintptr_t>(p.plan.lw.p));
    if (!b->exec || key != b->graph_key) {
        drop_graph(b);
        // one run of the path launches outside the capture, so that whatever they allocate or set
        // on first use is in place before it
        if (!b->paths.empty()) BCHECK(enqueue_paths(b));
        BCHECK(bcuda(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "batch capture"));
        int rc = enqueue(b, D, off, smem, fold_total, true);
        if (rc == SPRING_OK) rc = enqueue_paths(b);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (rc != SPRING_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        BCHECK(bcuda(b, e, "batch capture"));
        b->graph = graph;
        BCHECK(bcuda(b, cudaGraphInstantiate(&b->exec, b->graph, 0), "batch graph"));
        b->graph_key = key;
    }
    BCHECK(bcuda(b, cudaEventRecord(b->ev0, b->stream), "batch timing"));
    BCHECK(bcuda(b, cudaGraphLaunch(b->exec, b->stream), "batch graph launch"));
    b->work[0].c->launches += 2;
    BCHECK(run_tc_requests(b));
    BCHECK(bcuda(b, cudaEventRecord(b->ev1, b->stream), "batch timing"));
    BCHECK(join_out(b));
    BCHECK(bcuda(b, cudaEventSynchronize(b->ev1), "batch run"));
    float t = 0.0f;
    BCHECK(bcuda(b, cudaEventElapsedTime(&t, b->ev0, b->ev1), "batch timing"));
    b->last_ms = t;
    return SPRING_OK;
}

int spring_batch_result(spring_batch* b, int index, double* lw, double* p3_q0, double* ms) {
    if (!b) return SPRING_ERR_ARG;
    b->err.clear();
    if (index < 0 || index >= (int)b->work.size()) return bfail(b, SPRING_ERR_ARG, "no request %d", index);
    spring::Guard g(b->device);
    const auto& w = b->work[index];
    spring_ctx* c = w.c;
    if (!c->d_lw_tmp.p || !c->d_p3.p) return bfail(b, SPRING_ERR_STATE, "the batch has not run");
    if (lw && spring::lw_out(c, c->d_lw_tmp.p, w.q0, w.n_q0, lw) != SPRING_OK)
        return bfail(b, SPRING_ERR_CUDA, "%s", c->err.c_str());
    if (p3_q0 && spring::d2h(c, p3_q0, c->d_p3.p + (size_t)w.q0 * c->ndof, sizeof(double) * w.n_q0 * c->ndof,
                             "P3_q0") != SPRING_OK)
        return bfail(b, SPRING_ERR_CUDA, "%s", c->err.c_str());
    if (ms) *ms = b->last_ms;
    return SPRING_OK;
}

}  // extern "C"
