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

// Momentum-conserving pairs of every q0 of one set of q0 points (the point-group
// irreducible set of kappa.x, or the time-reversal set of kappa_iter.x).
struct PairSet {
    int n0 = 0;
    const int* q0_int = nullptr;  // [n0][3] device, not owned
    const int* q0_grid = nullptr; // [n0] grid index of each q0 (device) or null
    DBuf<int> partner;            // [q0][q1] partner grid index (0-based)
    DBuf<int> pairoff;            // [n0 + 1]
    DBuf<int2> pairs;             // (g1, g2) 0-based, grouped by q0
    DBuf<int> pair_q0;            // q0 of each pair
    DBuf<int> pairpos;            // [q0][q1] exclusive-scan position of each representative
    mutable std::vector<int> h_pairoff;  // host copy of pairoff, read on first use (pairoff_host)
    mutable bool h_ok = false;
    int cap = 0;                  // pairs and pair_q0 hold this many entries
    bool done = false;
    int gen = 0;                  // bumped every time the lists are rebuilt
};

// The q0 side of the V3 kernel: integer q0 vectors and the phonons of each q0.
struct Q0View {
    const int* q0_int;      // [n0][3]
    const int* q0_grid;     // null: phonons indexed by q0; else by q0_grid[q0]
    const double2* evec;
    const double* omega;
    const double* oneby;
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

// The surrogate network (k_mlp.cu): parameters, gradient, Adam moments, activations.
struct Mlp {
    DBuf<float> p, g, m, v, act, scal;
    int cap = 0;          // rows the activation buffers hold
    long long step = 0;   // Adam step
    bool set = false;
};

// Dipole-dipole term (spring_set_dipole, k_ewald.cu): the q-independent tables on the device.
struct EwaldDev {
    bool on = false, even = false;  // even: a G or R mesh of even size (no time-reversal shortcut)
    int ng = 0, nr = 0, gmesh[3] = {0, 0, 0}, rmesh[3] = {0, 0, 0};
    double lmb = 0.0, vol = 0.0, eps[9] = {};
    DBuf<double> g, r, hz, tau, z;
    DBuf<double2> cc, dd;
};

// Point-defect scattering (spring_set_point_defect, k_pdef.cu).
struct PointDefectDev {
    bool on = false, mat_inv_full = true, optc_therm = true;
    int nq = 0;
    double rho = 0.0;
    DBuf<double> vfc, vm, qpnt, w2;
    DBuf<int> qint, tet, inc, gamma0;
    DBuf<double2> wgt, G, te0;
    Phonons ph;
};

}  // namespace spring

struct spring_ctx {
    int device = 0;
    int nb = 0, ndof = 0;
    int mesh[3] = {0, 0, 0};
    int nq = 0, nq0 = 0, nT = 1;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int* h_pin = nullptr;              // pinned host scratch for readbacks that overlap queued work
    size_t h_pin_n = 0;                // its size in ints
    cudaEvent_t ev_aux = nullptr;      // marks the end of such a readback
    // Pinned staging ring for host -> device copies: every upload copies the caller's bytes here on
    // the CPU before its cudaMemcpyAsync is queued, so no copy ever reads host memory the library
    // does not own.  Bytes are reused only after ev_stage (recorded behind the last staged copy)
    // has completed.
    char* h_stage = nullptr;
    size_t h_stage_cap = 0, h_stage_off = 0;
    cudaEvent_t ev_stage = nullptr;
    bool stage_pending = false;
    cudaStream_t stream2 = nullptr;    // side stream for work that overlaps the main stream's
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::string err;
    long long launches = 0;
    int precision = SPRING_FP64;
    bool force_generic_v3 = false;  // spring_set_option(SPRING_OPT_GENERIC_V3): use the any-cell V3 kernel
    long long tc_max_spins = -1;    // spring_set_option(SPRING_OPT_WAIT_POLLS); -1: the kernels' default
    bool fp64_prescreen = false;    // spring_set_option(SPRING_OPT_FP64_PRESCREEN)

    // per-launch CUDA-event records (spring_set_profiling)
    struct ProfRec {
        std::string name;
        cudaEvent_t start, stop;
    };
    bool profiling = false;
    std::vector<ProfRec> prof;
    cudaEvent_t prof_pending = nullptr;

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

    // FC3: [mu][N1][N2][alpha][beta][gamma] (Fortran memory order), zero beyond atm_num
    bool fc3_set = false;
    int na3 = 0;
    spring::DBuf<double> d_fc3;
    spring::DBuf<double> d_fc3_posr;  // [mu][N][3]  Cartesian cell vector
    spring::DBuf<int> d_fc3_btyp;     // [mu][N] 0-based basis index
    spring::DBuf<int> d_fc3_off;      // [mu][nb+1] first slot of each basis atom (slots grouped by basis)

    // FC4: [mu][N1][N2][N3][a][b][c][d] (Fortran memory order), slots grouped by basis like FC3
    bool fc4_set = false;
    int na4 = 0;
    spring::DBuf<double> d_fc4;
    spring::DBuf<double> d_fc4_posr;  // [mu][N][3]
    spring::DBuf<int> d_fc4_btyp;     // [mu][N]
    spring::DBuf<int> d_fc4_off;      // [mu][nb+1]

    // mesh
    bool mesh_set = false;
    bool mesh_zc = true;           // zero-centred folding (kappa.x) or [0, N) (LineWidth.x)
    int mesh_shift[3] = {0, 0, 0};
    spring::DBuf<int> d_qint;      // [q][3]
    // time-reversal pairs of the grid (Gamma-centred meshes): partner of each point, points solved /
    // filled, for the mesh of tr_nq points
    spring::DBuf<int> d_tr_partner, d_tr_solve, d_tr_fill;
    int tr_nq = -1, tr_nsolve = 0, tr_nfill = 0;
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

    // 3-phonon pairs of the irreducible set and of the time-reversal set
    spring::PairSet ps_irr, ps_tr;
    // time-reversal set (kappa_iter.x): representatives, their F slots and signs
    int ntr = 0;
    spring::DBuf<int> d_tr_int;    // [ntr][3]
    spring::DBuf<int> d_tr_grid;   // [ntr] grid index
    spring::DBuf<int> d_tr_pos;    // [q] slot of each grid point
    spring::DBuf<int> d_tr_sgn;    // [q] +1 representative, -1 its inverse
    spring::DBuf<int> d_tr_deg;    // [ntr]
    spring::DBuf<int> d_neg;       // [q] grid index of -q
    spring::DBuf<double> d_wtr;    // cached W grids of the time-reversal set
    spring::DBuf<double> d_v4_rec;  // V4 tensor-core mode records (omega, 1/omega, n(T))
    spring::EwaldDev ew;
    spring::PointDefectDev pd;
    std::vector<double> h_fc2;     // host copies of FC2 (the point-defect perturbation)
    std::vector<int> h_fc2_idx, h_fc2_num;
    // sorted Gaussian BTE operator (k_bte.cu run_bte_gauss): rows, (k1, k2), (P, Q)
    spring::DBuf<int> d_bteg_row;
    spring::DBuf<int2> d_bteg_kk;
    spring::DBuf<double2> d_bteg_pq;
    long long bteg_n = 0;
    double bteg_sigma = 0.0;
    int bteg_gen = -1, bteg_pairs = -1, bteg_prec = -1;

    // four-phonon quartet lists (k_4ph.cu, opaque) and the tensor-core V4 buffers (k_v4tc.cu)
    void* e4 = nullptr;
    spring::DBuf<double2> d_v4_ph;    // [q][mu][8] phases
    spring::DBuf<float2> d_v4_etab;   // [q][nu c][s] m^-1/2 e
    spring::DBuf<float> d_v4_wf;      // [q][s] FP32 omega
    spring::DBuf<float2> d_v4_c;      // C of one q0
    spring::DBuf<short> d_v4_map;     // (mu, N2, N3) -> block entry
    spring::DBuf<uint4> d_v4_img;     // B images [q1][chunk][part]
    spring::DBuf<int> d_v4_cnt, d_v4_seg, d_v4_ntl, d_v4_toff, d_v4_stat;
    spring::DBuf<int4> d_v4_tiles;

    // scratch
    spring::DBuf<int> d_scan_tmp;
    spring::DBuf<double> d_w;      // W buffer for tetrahedron integration [slot][q1][s0][s1][s2]
    spring::DBuf<double> d_lw_all; // resident LW_Allq0 [T][q0][s]
    spring::DBuf<double> d_lw_tmp; // per-call output [T][q0][s]
    spring::DBuf<double> d_p3;     // per-call phase space [q0][s]
    spring::DBuf<double> d_kappa;  // [T][9] and mode [T][s][9]
    spring::DBuf<double> d_kap_part;  // per-block partial sums of the kappa kernel
    spring::DBuf<double> d_krn;    // [q0][s][9]
    spring::DBuf<double> d_rxyz;
    spring::DBuf<double> d_wiso;   // [slot][q1][s0][s1]

    // tensor-core V3 (spring_set_precision): operand tables and pair tiles grouped by q1
    spring::DBuf<uint16_t> d_tc_a;     // bf16 A operand images [q][hi, lo][mu]
    spring::DBuf<uint16_t> d_tc_b;     // bf16 B operand images [q1][hi, lo][mu]
    spring::DBuf<double> d_tc_q0;      // q0 mode records: e0' float2[6], omega, 1/omega (64 bytes each)
    spring::DBuf<double> d_tc_modes;   // grid mode records: omega, 1/omega, nBE[T] (padded to 4 doubles)
    spring::DBuf<int> d_tc_cnt_cta;    // status word of the tensor-core pass
    spring::DBuf<int> d_scr_sum;       // one-int readback scratch
    spring::DBuf<int> d_scr_rot, d_scr_map;  // spring_find_irr_q scratch: rotations, orbit map
    int tc_grid = 0;
    spring::DBuf<int> d_tc_entries;    // pair indices sorted by q1
    spring::DBuf<int4> d_tc_rec;       // (q0, q2, weight, q0 is Gamma) in that order
    spring::DBuf<int4> d_tc_tiles;     // (q1, first entry, count)
    int tc_ntiles = 0, tc_gen = -1, tc_q0 = -1, tc_n0 = -1, tc_nmax = 0, tc_ph_gen = -1;  // tile cache key
    int tc_set = -1;                   // q0 set of the cached tiles (0 irreducible, 1 time-reversal)
    spring::DBuf<double2> d_tr_ev;     // time-reversal q0 phonons gathered from the grid (tensor-core operator)
    spring::DBuf<double> d_tr_om, d_tr_ob;
    int tr_ph_gen = -1;
    int tc_npairs = 0;                 // pairs in those tiles
    float tc_rf = 0.0f;                // delta window the cached tiles were screened with
    bool tc_pending = false;           // tile count read back asynchronously, tiles not cut yet
    int ph_gen = 0;                    // bumped whenever the grid or irreducible phonons change
    // scratch kept between calls (the enumeration and the tile sort run every step)
    spring::DBuf<int> d_scr_rep, d_tc_keys, d_tc_keys_s, d_tc_vals, d_tc_cnt, d_tc_seg, d_tc_ntl, d_tc_toff;
    spring::DBuf<uint8_t> d_tc_sort;

    spring::Mlp mlp;
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
inline void free_pairs(PairSet& s) {
    dfree(s.partner); dfree(s.pairoff); dfree(s.pairs); dfree(s.pair_q0); dfree(s.pairpos);
    s.h_pairoff.clear();
    s.h_ok = false;
    s.done = false;
}
void free_phonons(Phonons& p);
int alloc_phonons(spring_ctx* c, Phonons& p, int n);
int h2d(spring_ctx* c, void* dst, const void* src, size_t bytes, const char* what);
int d2h(spring_ctx* c, void* dst, const void* src, size_t bytes, const char* what);
int zero(spring_ctx* c, void* dst, size_t bytes, const char* what);
int d2h_sum2(spring_ctx* c, const int* a, const int* b, int* out, const char* what);
// Host copy of a pair set's offsets (one readback after each enumeration, on first use).
int pairoff_host(spring_ctx* c, const PairSet& ps);
// Device -> pinned host copy of `bytes` ending in an event; pin_wait() waits for it.
int d2h_pin_async(spring_ctx* c, const void* src, size_t bytes, const char* what);
int pin_wait(spring_ctx* c, const char* what);
// Every kernel launch site calls launch_injected() first (fault injection and,
// when profiling, the start event) and launch_check() right after the launch
// (error check, launch count, stop event named after the kernel).
int launch_check(spring_ctx* c, const char* what);
bool launch_injected(spring_ctx* c);

// ---- kernels (host launchers), each defined in its own .cu -------------------
// k_mesh.cu
int run_make_mesh(spring_ctx* c, const int shift[3], int zero_centered);
int run_irr_map(spring_ctx* c, const int* d_rot, int nrot, int time_rev, int* d_map);
// k_phonon.cu
// gamma_mode: how the dipole term picks the Gamma direction (0: the next point of the list, 1: a
// fixed direction, for single points)
int run_phonons(spring_ctx* c, Phonons& ph, const double* d_q, int n, int gamma_mode = 0);
int set_dipole(spring_ctx* c, const double* atm_pos, const double* eps, const double* zstar, int decide,
               double prec_ew, double lmb, const int* gmesh, const int* rmesh, const int* sup_cell);
int set_point_defect(spring_ctx* c, const int* qmesh, int na_p, const int* num_p, const int* idx_p, const double* fc_p,
                     const double* mass_def, double rho, int mat_inv_full, int optc_therm);
int run_point_defect(spring_ctx* c, int i0_first, int n_q0, double* d_rate);
int run_point_defect_add(spring_ctx* c, int i0_first, int n_q0, const double* d_rate);
// make_tetrahedron for another mesh into the given buffers (qint [nq][3], qpnt [nq][3], tet [6 nq][4])
int run_make_mesh_on(spring_ctx* c, const int mesh[3], const int shift[3], int zc, int* d_qint, double* d_qpnt,
                     int* d_tet);
int launch_ewald(spring_ctx* c, const double* qa, int nqa, const int* list_a, int n_a, const double* qb, int nqb,
                 int n_b, int gamma_mode, const double2** dd_out);
int run_phonons_mesh(spring_ctx* c);  // grid + irreducible points (time reversal on Gamma-centred meshes)
// k_enum.cu
int run_enumerate3(spring_ctx* c, PairSet& ps);
int run_enumerate3_fortran(spring_ctx* c, int i0, int* d_allq1q2, int* d_perm, int* d_counts);
int run_exclusive_scan(spring_ctx* c, const int* d_in, int* d_out, int n);
// k_v3.cu
struct Pol { int lo[3], hi[3]; };
Q0View irr_view(spring_ctx* c);
int run_v3_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3);
int run_v3_wgrid(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, double* d_w);
// k_v3s.cu: specialised V3 for two-atom cells; *handled is false when the cell does not fit it
int launch_v3s(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, int epi, double sigma,
               const Pol* pol, double* lw, double* p3, double* w, bool* handled, const int* plist = nullptr,
               int nlist = 0);
int launch_v3s_bte(spring_ctx* c, const PairSet& ps, const Q0View& v, int q0_first, int n_q0, double sigma,
                   void* items, unsigned long long* ctr, long long cap, bool* handled);
// k_bteg.cu: iterative kappa with Gaussian deltas (the operator stored sparse in HBM)
int run_bte_gauss(spring_ctx* c, double sigma, double eps_k, int max_iter, double* h_kappa, double* h_kappa_rta,
                  int* h_iters, double* h_stats);
// k_v3tc.cu: the pairs of a q0 block with a mode triple inside the Gaussian's exp(-40) window (the
// tensor-core path's pre-screen), as a device list of pair indices and its length
int run_v3_prescreen(spring_ctx* c, int q0_first, int n_q0, double sigma, const int** d_list, int* n);
// k_v3tc.cu: tensor-core V3 + Gaussian sum (BF16 / BF16x3) for two-atom cells; *handled false otherwise
// k_v3tc.cu: entries of the Gaussian iterative-BTE operator (s3::BteEntry layout) over time-reversal
// q0 block [q0_first, q0_first + n_q0) on the tensor cores; *handled false when the cell or the
// precision (FP64) does not take it.  *ctr receives the entry count, which may exceed cap.
int run_v3tc_bte(spring_ctx* c, int q0_first, int n_q0, double sigma, void* entries, unsigned long long* ctr,
                 long long cap, bool* handled);
int run_v3tc_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const Pol& pol, double* d_lw, double* d_p3,
                   bool* handled);
// k_4ph.cu
int run_enumerate4_fortran(spring_ctx* c, int q0, int* d_all, int* d_perm, long long cap, long long* h_counts);
int run_lw4(spring_ctx* c, int q0_first, int n_q0, int delta_mode, double sigma, const int* pol4, double* d_rate);
int run_enum4_list(spring_ctx* c, int q0, const int4** d_quart, long long* nquart);
void free_enum4(spring_ctx* c);
// k_v4tc.cu: tensor-core V4 + Gaussian four-phonon rate (BF16 / BF16x3) for two-atom cells;
// *handled false when the cell or the precision does not take it
// h_mask: per q0 of the block, the branches s0 (bit s0) to compute; null for all
int run_v4tc_gauss(spring_ctx* c, int q0_first, int n_q0, double sigma, const int* h_mask, double* d_rate,
                   bool* handled);
// k_path.cu: LineWidth.x path mode; h_q0 (3, n_path) Cartesian, h_lw [T][p][s], h_omega [p][s]
int run_path(spring_ctx* c, int n_path, const double* h_q0, const int* h_zc, int delta_mode, double sigma,
             double* h_lw, double* h_omega);
// The same in three steps: path_prepare allocates every buffer of the run and uploads the points;
// path_enqueue queues its launches and memsets on c->stream (no allocation, copy from the host or
// wait on the host, so a stream capture may record it); path_fetch copies the results back.
struct PathPlan {
    int n_path = 0, slots = 0;
    DBuf<double> q0v, q1v, q2v, w, lw, p3;
    DBuf<int> zc, ex;
    Phonons php, ph2;
};
int path_prepare(spring_ctx* c, PathPlan& p, int n_path, const double* h_q0, const int* h_zc);
int path_enqueue(spring_ctx* c, PathPlan& p, int delta_mode, double sigma);
int path_fetch(spring_ctx* c, PathPlan& p, double* h_lw, double* h_omega);
void path_release(PathPlan& p);
int path_points(const double* G, int n_nodes, const double* q_high_sym, double* qpoints, double* dist, int* zc);
// k_mlp.cu: the surrogate network (row-major X[n][SPRING_MLP_INPUTS], y[n])
int mlp_num_params();
int run_mlp_init(spring_ctx* c, unsigned long long seed);
int run_mlp_set(spring_ctx* c, const float* params);
int run_mlp_loss_grad(spring_ctx* c, int n, const float* hX, const float* hy, float* loss, float* grad);
int run_mlp_train(spring_ctx* c, int n, const float* hX, const float* hy, int epochs, int batch, float lr,
                  unsigned long long seed, float* epoch_loss);
int run_mlp_predict(spring_ctx* c, int n, const float* hX, float* hy, int bf16);
void free_mlp(Mlp& m);
// k_bte.cu
int run_bte(spring_ctx* c, double eps_k, int max_iter, double* h_kappa, double* h_kappa_rta, int* h_iters);
// k_tetra.cu
int run_tetra3(spring_ctx* c, int q0_first, int n_q0, const double* d_w, const Pol& pol, double* d_lw, double* d_p3);
// LineWidth.x form: strict bounds, q2 phonons of vertex q1 from a table of `ntab` rows (row = slot * Nq + q1)
int run_tetra3_path(spring_ctx* c, int p_first, int n_slots, int n_path, const double* d_w, const double* om0,
                    const double* om2t, const double* nbe2t, long long ntab, double* d_lw, double* d_scratch);
int run_iso(spring_ctx* c, int q0_first, int n_q0, int delta_mode, double sigma, const double* g2, double* d_rate);
// k_kappa.cu
int run_axpy_lw(spring_ctx* c, double a, const double* d_x, double* d_y, int q0_first, int n_q0);
// api.cu: checks and prerequisites of a Gaussian linewidth3 request; [T][q0 range][s] slab to the host
int prepare_lw3(spring_ctx* c, int i0_first, int n_q0, const int* pol3, Pol* pol);
int lw_out(spring_ctx* c, const double* d_src, int q0_first, int n_q0, double* out);
int run_kappa_rta(spring_ctx* c, int symm, int nsym, const double* d_rxyz, int s_lo, int s_hi, double* d_kappa,
                  double* d_mode);

}  // namespace spring

#define SPRING_CHECK(expr)                  \
    do {                                    \
        int _rc = (expr);                   \
        if (_rc != SPRING_OK) return _rc;   \
    } while (0)
