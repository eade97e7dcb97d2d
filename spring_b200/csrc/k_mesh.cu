// Mesh, tetrahedra and the irreducible-point map on the device.
//  - make_tetrahedron (src/Kappa/Src/TetrahedronQ_m.f90:56-221): one thread
//    per grid point writes its folded address and Cartesian q; one thread per
//    mesh cell writes its six tetrahedra in the reference's vertex pattern.
//  - FindIrrQ's spglib call (TetrahedronQ_m.f90:261): each grid point maps to
//    the smallest grid index of its orbit under the reciprocal rotations W^T.
// Integer work; bound by writes to HBM (negligible next to the scattering path).
#include "spring_internal.cuh"

namespace spring {
namespace {

struct MeshArgs {
    int n0, n1, n2;
    double ru[9];  // Recp_cell_unit(r, c) = G(r, c)/mesh(c), stored ru[r*3+c]
    int shift[3];
    int zero_centered;
};

__device__ __forceinline__ int fold1(int v, int n, int zc) {
    if (zc) return v > n / 2 ? v - n : v;       // fold_indx (IndxChng_mod.f90:85-107)
    return v == n ? 0 : v;                       // MapAwayFromBZboundary (:110-135)
}

__device__ __forceinline__ int imod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

__global__ void k_grid_points(MeshArgs a, int* __restrict__ qint, double* __restrict__ qpnt) {
    const int nq = a.n0 * a.n1 * a.n2;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x) {
        int v[3] = {g % a.n0, (g / a.n0) % a.n1, g / (a.n0 * a.n1)};
        const int n[3] = {a.n0, a.n1, a.n2};
        for (int d = 0; d < 3; ++d) v[d] = fold1(v[d], n[d], a.zero_centered);
        for (int d = 0; d < 3; ++d) qint[3 * g + d] = v[d];
        for (int r = 0; r < 3; ++r) {
            // same operation order as the oracle: ((ru0*x0 + ru1*x1) + ru2*x2), no contraction
            double s = 0.0;
            for (int k = 0; k < 3; ++k)
                s = __dadd_rn(s, __dmul_rn(a.ru[r * 3 + k], (double)v[k] + (double)a.shift[k] * 0.5));
            qpnt[3 * g + r] = s;
        }
    }
}

__global__ void k_tetrahedra(MeshArgs a, int4* __restrict__ tet) {
    const int box[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0}, {0, 1, 0}};
    const int nq = a.n0 * a.n1 * a.n2;
    const int n[3] = {a.n0, a.n1, a.n2};
    for (int cidx = blockIdx.x * blockDim.x + threadIdx.x; cidx < nq; cidx += gridDim.x * blockDim.x) {
        int base[3] = {cidx % a.n0, (cidx / a.n0) % a.n1, cidx / (a.n0 * a.n1)};
        if (a.zero_centered)
            for (int d = 0; d < 3; ++d) base[d] = fold1(base[d], n[d], 1);
        int bt[8];
        for (int v = 0; v < 8; ++v) {
            int g = 0, mul = 1;
            for (int d = 0; d < 3; ++d) {
                int vf = fold1(box[v][d] + base[d], n[d], a.zero_centered);
                g += imod(vf, n[d]) * mul;
                mul *= n[d];
            }
            bt[v] = g;
        }
        // vertex pattern (1,5,2,4) (2,4,6,5) (8,4,6,5) (8,4,7,5) (7,4,3,5) (1,4,3,5)
        int4* o = tet + 6 * (size_t)cidx;
        o[0] = make_int4(bt[0], bt[1], bt[2], bt[3]);
        o[1] = make_int4(bt[2], bt[3], bt[4], bt[1]);
        o[2] = make_int4(bt[5], bt[3], bt[4], bt[1]);
        o[3] = make_int4(bt[5], bt[3], bt[6], bt[1]);
        o[4] = make_int4(bt[6], bt[3], bt[7], bt[1]);
        o[5] = make_int4(bt[0], bt[3], bt[7], bt[1]);
    }
}

__global__ void k_irr_map(int n0, int n1, int n2, const int* __restrict__ qint, const int* __restrict__ rot, int nrot,
                          int time_rev, int* __restrict__ map) {
    extern __shared__ int srot[];
    for (int i = threadIdx.x; i < 9 * nrot; i += blockDim.x) srot[i] = rot[i];
    __syncthreads();
    const int nq = n0 * n1 * n2;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nq; g += gridDim.x * blockDim.x) {
        const int a0 = qint[3 * g], a1 = qint[3 * g + 1], a2 = qint[3 * g + 2];
        int best = g;
        for (int s = 0; s < nrot; ++s) {
            const int* W = srot + 9 * s;
            // reciprocal rotation W^T acting on the grid address
            int b0 = W[0] * a0 + W[3] * a1 + W[6] * a2;
            int b1 = W[1] * a0 + W[4] * a1 + W[7] * a2;
            int b2 = W[2] * a0 + W[5] * a1 + W[8] * a2;
            int gi = imod(b0, n0) + n0 * (imod(b1, n1) + n1 * imod(b2, n2));
            best = min(best, gi);
            if (time_rev) {
                gi = imod(-b0, n0) + n0 * (imod(-b1, n1) + n1 * imod(-b2, n2));
                best = min(best, gi);
            }
        }
        map[g] = best;
    }
}

MeshArgs mesh_args(spring_ctx* c, const int shift[3], int zc) {
    MeshArgs a;
    a.n0 = c->mesh[0];
    a.n1 = c->mesh[1];
    a.n2 = c->mesh[2];
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) a.ru[r * 3 + k] = c->G[r + 3 * k] / double(c->mesh[k]);
    for (int k = 0; k < 3; ++k) a.shift[k] = shift ? shift[k] : 0;
    a.zero_centered = zc;
    return a;
}

}  // namespace

int run_make_mesh(spring_ctx* c, const int shift[3], int zc) {
    MeshArgs a = mesh_args(c, shift, zc);
    const int threads = 256;
    const int blocks = (c->nq + threads - 1) / threads;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "make_mesh: injected launch failure");
    k_grid_points<<<blocks, threads, 0, c->stream>>>(a, c->d_qint.p, c->d_qpnt.p);
    SPRING_CHECK(launch_check(c, "k_grid_points"));
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "make_mesh: injected launch failure");
    k_tetrahedra<<<blocks, threads, 0, c->stream>>>(a, reinterpret_cast<int4*>(c->d_tetra.p));
    return launch_check(c, "k_tetrahedra");
}

int run_make_mesh_on(spring_ctx* c, const int mesh[3], const int shift[3], int zc, int* d_qint, double* d_qpnt,
                     int* d_tet) {
    MeshArgs a = mesh_args(c, shift, zc);
    a.n0 = mesh[0];
    a.n1 = mesh[1];
    a.n2 = mesh[2];
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) a.ru[r * 3 + k] = c->G[r + 3 * k] / mesh[k];
    const int nq = mesh[0] * mesh[1] * mesh[2];
    const int threads = 256, blocks = (nq + threads - 1) / threads;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "make_mesh: injected launch failure");
    k_grid_points<<<blocks, threads, 0, c->stream>>>(a, d_qint, d_qpnt);
    SPRING_CHECK(launch_check(c, "k_grid_points"));
    k_tetrahedra<<<blocks, threads, 0, c->stream>>>(a, reinterpret_cast<int4*>(d_tet));
    return launch_check(c, "k_tetrahedra");
}

int run_irr_map(spring_ctx* c, const int* d_rot, int nrot, int time_rev, int* d_map) {
    const int threads = 256;
    const int blocks = (c->nq + threads - 1) / threads;
    if (launch_injected(c)) return fail(c, SPRING_ERR_INJECTED, "irr_map: injected launch failure");
    k_irr_map<<<blocks, threads, sizeof(int) * 9 * nrot, c->stream>>>(c->mesh[0], c->mesh[1], c->mesh[2], c->d_qint.p,
                                                                     d_rot, nrot, time_rev, d_map);
    return launch_check(c, "k_irr_map");
}

}  // namespace spring
