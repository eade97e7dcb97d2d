// Internal declarations shared by the translation units of libspring_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/spring_gpu.h"

namespace spring {

// Unit factors of src/Kappa/Src/constants.f90:27-63 (same literal expressions).
constexpr double PI = 3.141592653589793;  // 4*atan(1) in FP64
constexpr double ONEBYSQRT2PI = 0.3989422804014327;
constexpr double CMP_PREC = 1.0e-8;
constexpr double EPS_F32 = 9.99999993922529029e-09;  // 1.0E-8 default-real literal widened to dp
constexpr double ONEBYSIX = 0.16666666666666666;
constexpr int MAX_NB = 8;
constexpr int MAX_NDOF = 3 * MAX_NB;

struct HostConst {
    double wTHz, vg_ms, BEConv, Sctr3THz2, Sctr4THz2, kW_m_k;
};
HostConst host_constants();

// Device buffer with an owner.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
};

struct Phonons {
    int n = 0;                       // number of q points
    DBuf<double2> evec;              // [q][s][row]  (Fortran Evec(row,s,q))
    DBuf<double> omega;              // [q][s]
    DBuf<double> oneby;              // [q][s]
    DBuf<double> nbe;                // [T][q][s]
    DBuf<double> vel;                // [q][s][3]
    bool set = false;
};

}  // namespace spring

struct spring_ctx {
    int device = 0;
    int nb = 0, ndof = 0;
    int mesh[3] = {0, 0, 0};
    int nq = 0, nq0 = 0, nT = 1;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    int precision = SPRING_FP64;

    // fault injection
    int inject_kind = -1;
    long long inject_n = 0, inject_seen[3] = {0, 0, 0};

    // crystal
    bool crystal_set = false;
    double latvec[9] = {0}, G[9] = {0}, vol = 0.0;
    std::vector<double> mass;
    spring::DBuf<double> d_mass_rs;  // 1/sqrt(mass)

    // FC2
    bool fc2_set = false;
    int na2 = 0;
    spring::DBuf<double> d_fc2;      // [mu][N][alpha][beta]
    spring::DBuf<int> d_fc2_idx;     // [mu][N][4]
    spring::DBuf<int> d_fc2_num;

    // FC3: kernel layout [mu][N2*3+gamma][(N1*3+alpha)*3+beta]  (zero padded to na3)
    bool fc3_set = false;
    int na3 = 0;
    spring::DBuf<double> d_fc3t;
    spring::DBuf<double> d_fc3_posr;  // [mu][N][3]  Cartesian cell vector
    spring::DBuf<int> d_fc3_btyp;     // [mu][N] 0-based basis index

    // mesh
    bool mesh_set = false;
    spring::DBuf<int> d_qint;      // [q][3]
    spring::DBuf<double> d_qpnt;   // [q][3]
    spring::DBuf<int> d_tetra;     // [t][4] 0-based grid indices
    bool irr_set = false;
    std::vector<int> h_irr_int, h_pos, h_mult;
    spring::DBuf<int> d_irr_int;   // [q0][3]
    spring::DBuf<double> d_irr_q;  // [q0][3]
    spring::DBuf<int> d_mult;
    spring::DBuf<int> d_pos;       // [q] 1-based irreducible slot of each grid point

    // phonons
    std::vector<double> temps;
    spring::DBuf<double> d_temps;
    spring::Phonons ph_grid, ph_irr;

    // 3-phonon enumeration, all irreducible points
    bool enum3_done = false;
    spring::DBuf<int> d_partner;   // [q0][q1] partner grid index (0-based)
    spring::DBuf<int> d_pairoff;   // [nq0+1]
    spring::DBuf<int2> d_pairs;    // (g1, g2) 0-based
    spring::DBuf<int> d_pair_q0;   // q0 of each pair
    spring::DBuf<int> d_pairpos;   // [q0][q1] exclusive-scan position of each representative
    std::vector<int> h_pairoff;

    // scratch
    spring::DBuf<int> d_scan_tmp;
    spring::DBuf<double> d_w;      // W buffer for tetrahedron integration [slot][q1][s0][s1][s2]
    spring::DBuf<double> d_lw_all; // resident LW_Allq0 [T][q0][s]
    spring::DBuf<double> d_lw_tmp; // per-call output [T][q0][s]
    spring::DBuf<double> d_p3;     // per-call phase space [q0][s]
    spring::DBuf<double> d_kappa;  // [T][9] and mode [T][s][9]
    spring::DBuf<double> d_krn;    // [q0][s][9]
    spring::DBuf<double> d_rxyz;
    spring::DBuf<double> d_wiso;   // [slot][q1][s0][s1]
};

namespace spring {

// error helpers (set ctx->err and return the status)
int fail(spring_ctx* c, int code, const char* fmt, ...);
int cuda_fail(spring_ctx* c, cudaError_t e, const char* what);

// allocation / copies with fault injection, all on ctx->stream
int dalloc_bytes(spring_ctx* c, void** p, size_t bytes, const char* what);
template <class T>
int dalloc(spring_ctx* c, DBuf<T>& b, size_t n, const char* what) {
    if (b.p && b.n >= n) return SPRING_OK;
    if (b.p) { cudaFree(b.p); b.p = nullptr; b.n = 0; }
    if (n == 0) n = 1;
    int rc = dalloc_bytes(c, (void**)&b.p, n * sizeof(T), what);
    if (rc == SPRING_OK) b.n = n;
    return rc;
}
template <class T>
void dfree(DBuf<T>& b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
}
int h2d(spring_ctx* c, void* dst, const void* src, size_t bytes, const char* what);
int d2h(spring_ctx* c, void* dst, const void* src, size_t bytes, const char* what);
int zero(spring_ctx* c, void* dst, size_t bytes, const char* what);
int launch_check(spring_ctx* c, const char* what);  // counts launches, checks cudaGetLastError
bool launch_injected(spring_ctx* c);

// ---- kernels (host launchers), each defined in its own .cu -------------------
// k_mesh.cu
int run_make_mesh(spring_ctx* c, const int shift[3], int zero_centered);
int run_irr_map(spring_ctx* c, const int* d_rot, int nrot, int time_rev, int* d_map);
// k_phonon.cu
int run_phonons(spring_ctx* c, Phonons& ph, const double* d_q, int n);
// k_enum.cu
int run_enumerate3(spring_ctx* c);
int run_enumerate3_fortran(spring_ctx* c, int i0, int* d_allq1q2, int* d_perm, int* d_counts);
int run_exclusive_scan(spring_ctx* c, const int* d_in, int* d_out, int n);
// k_v3.cu
struct Pol { int lo[3], hi[3]; };
int run_v3_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3);
int run_v3_wgrid(spring_ctx* c, int q0_first, int n_q0, double* d_w);
// k_tetra.cu
int run_tetra3(spring_ctx* c, int q0_first, int n_q0, const double* d_w, const Pol& pol, double* d_lw, double* d_p3);
int run_iso(spring_ctx* c, int q0_first, int n_q0, int delta_mode, double sigma, const double* g2, double* d_rate);
// k_kappa.cu
int run_axpy_lw(spring_ctx* c, double a, const double* d_x, double* d_y, int q0_first, int n_q0);
int run_kappa_rta(spring_ctx* c, int symm, int nsym, const double* d_rxyz, int s_lo, int s_hi, double* d_kappa,
                  double* d_mode);

}  // namespace spring

#define SPRING_CHECK(expr)                  \
    do {                                    \
        int _rc = (expr);                   \
        if (_rc != SPRING_OK) return _rc;   \
    } while (0)
