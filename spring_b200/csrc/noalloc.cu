// spring_linewidth3_tetra_noalloc: the 3-phonon tetrahedron linewidth of one q0
// with all of its scratch in a fixed device array of this library instead of
// device memory obtained at call time.
//
// Some callers cannot let a library call cudaMalloc: hosts whose device memory is
// owned by another allocator (a framework's caching pool, or a pool reserved up
// front by the host program), and pipelines that must not pay the device-wide
// synchronisation that cudaMalloc/cudaFree may imply between queued kernels.
// This entry point allocates nothing.  Its scratch (the W grid of the q0 and the
// accumulation slabs of the delta sum) lives in `g_noalloc_scratch` below; the
// caller passes the context (whose inputs were loaded beforehand) and the device
// buffers that receive the results.
//
// Limits and sharing:
//   - capacity: Nq*Ndof^3 + (n_temps + 1)*Nq0*Ndof doubles must not exceed
//     NOALLOC_CAPACITY (2^21 doubles = 16 MiB), e.g. a 2-atom cell up to about
//     9,700 q-points (21^3);
//   - the array is allocated when a GPU loads the library and is held until exit;
//   - every call shares the one array and leaves its contents behind; the slabs
//     that accumulate are cleared at the start of each call, and the W grid is
//     rewritten completely, so nothing depends on the previous call;
//   - calls whose GPU work overlaps (different streams or host threads) race on
//     the array and must be serialised by the caller;
//   - the first call on each device looks the array's address up
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture.
#include <mutex>

#include "spring_internal.cuh"

namespace spring {
namespace {

constexpr size_t NOALLOC_CAPACITY = (size_t)1 << 21;  // doubles

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_CAPACITY];

constexpr int MAX_DEVICES = 64;
std::mutex g_addr_mutex;
double* g_addr[MAX_DEVICES] = {nullptr};

// Device address of g_noalloc_scratch on device `dev` (looked up once, with `dev` current).
int scratch_address(spring_ctx* c, int dev, double** out) {
    if (dev < 0 || dev >= MAX_DEVICES) return fail(c, SPRING_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return SPRING_OK;
}

}  // namespace
}  // namespace spring

using namespace spring;

extern "C" int spring_linewidth3_tetra_noalloc(spring_ctx* c, int i0, const int* pol3, double* d_lw, double* d_p3) {
    if (!c) return SPRING_ERR_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != c->device) cudaSetDevice(c->device);
    c->err.clear();
    int rc = SPRING_OK;
    do {
        if (!d_lw || !d_p3) { rc = fail(c, SPRING_ERR_ARG, "d_lw and d_p3 must be device buffers"); break; }
        if (!c->irr_set || i0 < 1 || i0 > c->nq0) { rc = fail(c, SPRING_ERR_ARG, "i0 out of range or no irreducible set"); break; }
        if (!c->fc3_set || !c->mesh_set || !c->ph_grid.set || !c->ph_irr.set) {
            rc = fail(c, SPRING_ERR_STATE, "FC3, mesh and phonons must be loaded first");
            break;
        }
        if (!c->ps_irr.done) {
            rc = fail(c, SPRING_ERR_STATE, "pairs not enumerated: call spring_prepare3 first (it allocates)");
            break;
        }
        const size_t n = c->ndof;
        const size_t wsize = (size_t)c->nq * n * n * n;
        const size_t lsize = (size_t)c->nT * c->nq0 * n, psize = (size_t)c->nq0 * n;
        if (wsize + lsize + psize > NOALLOC_CAPACITY) {
            rc = fail(c, SPRING_ERR_UNSUPPORTED,
                      "no-alloc scratch holds %zu doubles; this mesh needs %zu (Nq*Ndof^3 + (n_temps+1)*Nq0*Ndof)",
                      NOALLOC_CAPACITY, wsize + lsize + psize);
            break;
        }
        Pol pol;
        for (int k = 0; k < 3; ++k) {
            pol.lo[k] = pol3 ? pol3[2 * k] - 1 : 0;
            pol.hi[k] = pol3 ? pol3[2 * k + 1] - 1 : (int)n - 1;
            if (pol.lo[k] < 0 || pol.hi[k] >= (int)n || pol.lo[k] > pol.hi[k]) {
                rc = fail(c, SPRING_ERR_ARG, "pol3 column %d out of range", k + 1);
                break;
            }
        }
        if (rc != SPRING_OK) break;
        double* base = nullptr;
        if ((rc = scratch_address(c, c->device, &base)) != SPRING_OK) break;
        double* w = base;
        double* lw = base + wsize;
        double* p3 = lw + lsize;
        const int q0 = i0 - 1;
        cudaError_t e = cudaMemsetAsync(lw, 0, sizeof(double) * (lsize + psize), c->stream);
        if (e != cudaSuccess) { rc = cuda_fail(c, e, "clear no-alloc slabs"); break; }
        if ((rc = run_v3_wgrid(c, c->ps_irr, irr_view(c), q0, 1, w)) != SPRING_OK) break;
        if ((rc = run_tetra3(c, q0, 1, w, pol, lw, p3)) != SPRING_OK) break;
        // lw slab [T][q0][s] -> caller's [T][s];  p3 [q0][s] -> caller's [s]
        e = cudaMemcpy2DAsync(d_lw, n * sizeof(double), lw + (size_t)q0 * n, (size_t)c->nq0 * n * sizeof(double),
                              n * sizeof(double), c->nT, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_p3, p3 + (size_t)q0 * n, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) { rc = cuda_fail(c, e, "copy no-alloc results"); break; }
    } while (0);
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    return rc;
}
