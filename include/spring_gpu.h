/*
 * spring_gpu.h — C ABI of the B200 phonon-scattering library (libspring_b200.so).
 *
 * Replaces the hot path of SPRING's kappa.x / kappa_iter.x / LineWidth.x:
 * the per-q0 loop body of src/Kappa/Src/main.f90:552-715 and the kappa
 * stage main.f90:734-751.  A Fortran host binds these entry points with
 * iso_c_binding interfaces (bind(C), explicit-shape dummies, value scalars).
 *
 * Conventions
 *  - Every call returns an int status (SPRING_OK == 0); spring_last_error()
 *    gives the message of the last failure on that context.  Nothing throws.
 *  - Arrays are the reference's Fortran arrays, column-major, passed as plain
 *    pointers; the shape of each is written in Fortran order next to it.
 *  - Indices that cross the ABI (q-point / grid / quartet numbers) are 1-based.
 *  - complex(c_double_complex) arrays are interleaved (re, im) doubles.
 *  - The host keeps ownership of its arrays: the library copies inputs into
 *    device memory it owns and copies results back before returning.
 *  - Output pointers documented as optional may be NULL: the result then stays
 *    resident on the device for the next call (e.g. linewidths -> kappa).
 *  - A context is used by one host thread at a time.
 *  - Units are the reference's (src/Kappa/Src/constants.f90): omega in rad/ps,
 *    force constants in eV/A^n, masses in amu, kappa in W/m/K.
 */
#ifndef SPRING_GPU_H
#define SPRING_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spring_ctx spring_ctx;

/* status codes */
#define SPRING_OK 0
#define SPRING_ERR_ARG 1         /* invalid argument (NULL, size, range) */
#define SPRING_ERR_STATE 2       /* a required input has not been set */
#define SPRING_ERR_CUDA 3        /* CUDA runtime error (message has the CUDA text) */
#define SPRING_ERR_ALLOC 4       /* device allocation failed */
#define SPRING_ERR_UNSUPPORTED 5 /* valid request this build does not handle */
#define SPRING_ERR_INJECTED 6    /* failure injected by spring_debug_inject_fault */
#define SPRING_ERR_TIMEOUT 7     /* a bounded device-side wait ran out; the kernel stopped, the context stays usable */

/* delta-function schemes */
#define SPRING_DELTA_GAUSS 0 /* Gaussian smearing, ThirdOrder_m.f90:442-543 */
#define SPRING_DELTA_TETRA 1 /* linear tetrahedron, ThirdOrder_m.f90:169-275 */

/* arithmetic of the V3/V4 contractions (deltas, rates and kappa stay FP64) */
#define SPRING_FP64 0   /* FP64 CUDA cores, the reference's arithmetic */
#define SPRING_BF16 1   /* tcgen05 tensor cores, BF16 operands, FP32 accumulation */
#define SPRING_BF16X3 2 /* as SPRING_BF16 with hi+lo BF16 splits (compensated, about FP32 accuracy) */

typedef struct {
    int nbasis;  /* Nb: atoms in the unit cell (Ndof = 3*Nb), at most 8 */
    int mesh[3]; /* q-mesh (AnhInfo qmesh) */
    int n_temps; /* number of temperatures evaluated together (>= 1) */
    int device;  /* CUDA device ordinal; -1 = the calling thread's current device */
} spring_dims;

/* ---- context ---------------------------------------------------------- */
int spring_ctx_create(spring_ctx** ctx, const spring_dims* dims);
int spring_ctx_destroy(spring_ctx* ctx);
const char* spring_last_error(const spring_ctx* ctx);
/* Use the caller's CUDA stream (cudaStream_t) for all work; NULL restores the
 * context's own stream. */
int spring_set_stream(spring_ctx* ctx, void* cuda_stream);
int spring_synchronize(spring_ctx* ctx);
/* Number of launches of this library's kernels since the context was created. */
int spring_kernel_launches(const spring_ctx* ctx, long long* count);

/* ---- crystal and force constants (L1/L2 inputs) ------------------------ */
/* cell%init_data, src/Kappa/Src/unit_mod.f90:64-209: latvec(3,3) columns are
 * the lattice vectors (A); mass(Nb) per basis atom (amu).  Computes the cell
 * volume and the reciprocal vectors G like the reference. */
int spring_set_crystal(spring_ctx* ctx, const double* latvec, const double* mass);

/* Dipole-dipole (Ewald) term of D(q) for polar crystals (LongEw = &FCInfo Force_dd):
 * EwaldParam%set_EwaldParam (src/Kappa/Src/EwaldParam.f90) with &AtmInfo atm_pos(3,Nb),
 * dielec(3,3), BornZ(3,3,Nb), &CrystalInfo Sup_Cell(3) and &EwaldInfo decide_EwParam, prec_Ew,
 * Lmb, Gmesh(3), Rmesh(3) (Gmesh and Lmb are used only when decide_ew_param = 0; sup_cell NULL
 * = 5 5 5).  The phonons computed afterwards add DynMatgv_Ew (DynaMat_mod.f90:285-380), and
 * DynMat_NA with finite-difference velocities at q = 0 (get_phonon, :548-590).  dielec = NULL
 * switches the term off.  Needs spring_set_crystal; at most 8 basis atoms. */
int spring_set_dipole(spring_ctx* ctx, const double* atm_pos, const double* dielec, const double* born_z,
                      int decide_ew_param, double prec_ew, double lmb, const int* gmesh, const int* rmesh,
                      const int* sup_cell);
/* The parameters in use: on (0/1), Lmb, Gmesh(3), number of R and G points (NULL allowed). */
int spring_get_dipole(spring_ctx* ctx, int* on, double* lmb, int* gmesh, int* n_r, int* n_g);

/* Point-defect scattering (&PointDefInfo, ReadPointDefVar src/Kappa/Src/Helper_m.f90:135-307):
 * the perturbed FC2 of the defect cell (IFC2_file_pd: na2_pd, atm_num, atm_indx, fc2 in the
 * spring_set_fc2 layout), Mass_def(Nb) per basis atom (the pristine mass where no defect sits),
 * rho_def (defects per A^3), MatInvFull and OptcTherm (0/1), and qMesh_pd(3), the mesh of the
 * Green's-function tetrahedron integration.  Builds PerturbationMatrix
 * (point_defect_m.f90:40-108), the defect mesh (make_tetrahedron, zero-centred, the run's shift)
 * and its phonons.  Call after spring_set_fc2 (and spring_set_dipole) and spring_make_mesh.
 * qmesh_pd = NULL switches it off. */
int spring_set_point_defect(spring_ctx* ctx, const int* qmesh_pd, int na2_pd, const int* num_pd, const int* idx_pd,
                            const double* fc2_pd, const double* mass_def, double rho_def, int mat_inv_full,
                            int optc_therm);
/* ScatterRatePointDefect (point_defect_m.f90:139-376) for irreducible points i0_first ..
 * i0_first + n_q0 - 1 (1-based): rate(Ndof, n_q0) = 1/tau (NULL allowed; the Scatter_pd dataset);
 * add != 0 also adds 0.5 rate to the resident LW_Allq0 at every temperature (main.f90:685). */
int spring_linewidth_pd(spring_ctx* ctx, int i0_first, int n_q0, double* rate, int add);

/* FC2type%set_FC2, src/Kappa/Src/FC2_mod.f90:46-65:
 * atm_num(Nb), atm_indx(4,na2,Nb) = (cell R1,R2,R3, basis index), fc2(1,3,3,na2,Nb). */
int spring_set_fc2(spring_ctx* ctx, int na2, const int* atm_num, const int* atm_indx, const double* fc2);

/* FC3type%set_FC3, src/Kappa/Src/FC3_mod.f90:49-94: atm_indx(4,na3,Nb),
 * fc3(3,3,3,na3,na3,Nb) = (gamma,beta,alpha,N2,N1,mu). */
int spring_set_fc3(spring_ctx* ctx, int na3, const int* atm_num, const int* atm_indx, const double* fc3);

/* FC4type%set_FC4, src/Kappa/Src/FC4_mod.f90:46-97: atm_indx(4,na4,Nb),
 * fc4(3,3,3,3,na4,na4,na4,Nb) = (delta,gamma,beta,alpha,N3,N2,N1,mu). */
int spring_set_fc4(spring_ctx* ctx, int na4, const int* atm_num, const int* atm_indx, const double* fc4);

/* ---- mesh and irreducible q-points (L3) -------------------------------- */
/* q_tetrahedron%make_tetrahedron, src/Kappa/Src/TetrahedronQ_m.f90:56-221.
 * zero_centered = 1 folds to [-N/2+1, N/2] (kappa.x), 0 keeps [0, N) (LineWidth.x).
 * Outputs (optional): q_pnt_int(3,Nq), q_pnt(3,Nq), tetrahedrons(4,6*Nq). */
int spring_make_mesh(spring_ctx* ctx, const int* shift, int zero_centered, int* q_pnt_int, double* q_pnt,
                     int* tetrahedrons);

/* q_tetrahedron%FindIrrQ, TetrahedronQ_m.f90:224-331 (spglib's
 * spg_get_ir_reciprocal_mesh for a Gamma-centred mesh, then unique_sort and
 * FindPositionAndMultiplicity).  rotations(3,3,nrot) is the integer array
 * spg_get_symmetry fills (src/Kappa/Src/Symmetry_m.f90:84): its memory is
 * spglib's row-major W with x' = W x on fractional coordinates (the reference
 * transposes it to build Rxyz, :92-97).  Outputs: *nq0, irr_q_pnt_int(3,Nq)
 * (first nq0 columns used), pos(Nq) (1-based), multiplicity(Nq) (first nq0). */
int spring_find_irr_q(spring_ctx* ctx, int nrot, const int* rotations, int time_rev, int* nq0,
                      int* irr_q_pnt_int, int* pos, int* multiplicity);

/* ---- harmonic phonons (L4) -------------------------------------------- */
/* Phon%set_Phon_mp + get_phonon, src/Kappa/Src/phonon_mod.f90:156-313 and
 * DynaMat_mod.f90:486-709, for the grid and the irreducible set, every
 * temperature, on the device (batched FP64 Hermitian eigensolver).
 * temps(n_temps) in K; freq_cut is the -omegacut value (stored, not used on this path). */
int spring_compute_phonons(spring_ctx* ctx, const double* temps, double freq_cut);

/* Load phonons computed by the host (e.g. with LAPACK zheevd) instead.
 * which = 0: the Nq grid points; which = 1: the Nq0 irreducible points; which = 2: the
 * point-defect mesh (after spring_set_point_defect; evec and omega only, the rest may be NULL:
 * ph_pd of the reference, whose rates depend on the eigenvector gauge at degenerate levels).
 * evec(2,Ndof,Ndof,n) interleaved complex Evec(row,s,q); omega(Ndof,n);
 * onebyomega(Ndof,n); nbe(Ndof,n,n_temps); grp_vel(3,Ndof,n).  temps(n_temps). */
int spring_set_phonons(spring_ctx* ctx, int which, const double* temps, const double* evec, const double* omega,
                       const double* onebyomega, const double* nbe, const double* grp_vel);
/* Copy the device phonons back (any pointer may be NULL). */
int spring_get_phonons(spring_ctx* ctx, int which, double* evec, double* omega, double* onebyomega, double* nbe,
                       double* grp_vel);

/* ---- enumeration (L5) -------------------------------------------------- */
/* MomentumConsrv3rd, src/Kappa/Src/QuasiMomentumConsrv3rd_m.f90:13-158, for
 * q0 = irreducible point i0 (1-based), without the count assertions
 * (:148-153).  Allq1q2(4,Nq), q1q2_permuted(2,Nq) (first counts[0] columns),
 * counts = (pairs, total_count).  Outputs are bit-identical to the reference
 * algorithm's, on every mesh. */
int spring_enumerate3(spring_ctx* ctx, int i0, int* Allq1q2, int* q1q2_permuted, int* counts);

/* Enumerate the pairs of every irreducible q0 on the device (the same lists as
 * spring_enumerate3, kept resident for the scattering calls).  The scattering
 * calls run it on first use; calling it again recomputes it. */
int spring_prepare3(spring_ctx* ctx);

/* ---- three-phonon scattering ------------------------------------------ */
/* ScatterProbAllq1, src/Kappa/Src/ThirdOrder_m.f90:41-166: the W3 of every
 * grid q1 for q0 = i0; sctrq1(Ndof,Ndof,Ndof,Nq) = (s2,s1,s0,q1). */
int spring_scatter_w3(spring_ctx* ctx, int i0, double* sctrq1);

/* The 3-phonon linewidth of irreducible points i0_first .. i0_first+n_q0-1
 * at every temperature: V3 -> W -> delta sum, fused on the device.
 *   delta_mode SPRING_DELTA_TETRA: CalculateLwTetrahedron (ThirdOrder_m.f90:169-275);
 *   delta_mode SPRING_DELTA_GAUSS: CalculateLinewidth (ThirdOrder_m.f90:442-543),
 *     sigma in rad/ps (2 cm^-1 = 0.37673 rad/ps), branch start reset per q1.
 * pol3(2,3): Polarization3rd (Helper_m.f90:310-353) or NULL for all branches.
 * lw(Ndof,n_q0,n_temps) and p3_q0(Ndof,n_q0) are optional outputs; the
 * linewidth is also added to the context's resident LW_Allq0 (main.f90:584). */
int spring_linewidth3(spring_ctx* ctx, int i0_first, int n_q0, int delta_mode, double sigma, const int* pol3,
                      double* lw, double* p3_q0);

/* No counterpart in the reference.  The tetrahedron 3-phonon linewidth of one
 * irreducible point i0 (1-based) for callers that must not have the library
 * call cudaMalloc: hosts whose device memory belongs to another allocator, or
 * pipelines that cannot take the synchronisation cudaMalloc/cudaFree may imply.
 * Allocates nothing: its scratch is a fixed 16 MiB device array inside the
 * library (held by every GPU that loads it, until exit).  Limit:
 * Nq*Ndof^3 + (n_temps+1)*Nq0*Ndof <= 2^21 doubles (a 2-atom cell up to about
 * 21^3 q-points); larger meshes get SPRING_ERR_UNSUPPORTED.
 * Needs the inputs loaded and spring_prepare3 called beforehand.  d_lw (Ndof x
 * n_temps) and d_p3 (Ndof) are caller-owned DEVICE buffers; the context's
 * resident LW_Allq0 is not touched.  pol3 as in spring_linewidth3 (or NULL).
 * The first call on a device looks the array's address up; make it before any
 * stream capture.  All calls share the array: calls whose GPU work overlaps race
 * and must be serialised by the caller. */
int spring_linewidth3_tetra_noalloc(spring_ctx* ctx, int i0, const int* pol3, double* d_lw, double* d_p3);

/* Isotope scattering rate, CalculateIsoW + CalculateIsoLwTetra
 * (src/Kappa/Src/IsotopicScatter.f90:36-168); Gaussian form uses
 * delta(omega0 - omega1).  g2(Nb) mass variance.  rate(Ndof,n_q0,n_temps)
 * optional; 0.5*rate is added to the resident LW_Allq0 (main.f90:604). */
int spring_linewidth_iso(spring_ctx* ctx, int i0_first, int n_q0, int delta_mode, double sigma, const double* g2,
                         double* rate);

/* ---- four-phonon scattering ------------------------------------------- */
/* MomentumConsrv4th + Permutation4th, src/Kappa/Src/QuasiMomentumConsrv4th_m.f90:32-312,
 * for q0 = i0 (1-based): Allq1q2q3(3,Nq,Nq) = (permutation type, quartet
 * number, q3 grid index) of every ordered (q1, q2); q1q2q3_permuted(3,cap) the
 * grid indices of each quartet.  counts = (q1q2q3_count, total_count).  Both
 * arrays optional; more than cap quartets with a non-NULL q1q2q3_permuted is
 * SPRING_ERR_ARG.  Bit-identical to the reference algorithm on every mesh. */
int spring_enumerate4(spring_ctx* ctx, int i0, int* Allq1q2q3, int* q1q2q3_permuted, long long cap,
                      long long* counts);

/* The 4-phonon scattering rate of irreducible points i0_first .. +n_q0-1, every
 * temperature: quartets -> V4 -> W4 -> delta sum on the device.
 *   delta_mode SPRING_DELTA_TETRA: ScatterProbq1q2_per (FourthOrder_m.f90:286-473)
 *     + TetrahedronIntegration4th (Tetrahedron4th_sep.f90:37-425), every W read
 *     through the stored quartet with the reference's permutation of branches;
 *     holds one q0's quartet W (Nq^2/6 x Ndof^4 doubles) on the device.
 *   delta_mode SPRING_DELTA_GAUSS: the same three channels with
 *     delta(omega0 - M), W of each ordering from its quartet (build-side form).
 * Two-atom cells, na4 <= 8, n_temps <= 9.  pol4(2,4): Polarization4th or NULL.
 * rate(Ndof,n_q0,n_temps) optional; 0.5*rate is added to the resident LW_Allq0
 * (main.f90:661). */
int spring_linewidth4(spring_ctx* ctx, int i0_first, int n_q0, int delta_mode, double sigma, const int* pol4,
                      double* rate);

/* No counterpart in the reference.  The Gaussian 4-phonon rate of selected branches only: bit s-1 of
 * s0_mask(k) selects branch s of irreducible point i0_first + k - 1.  With the tensor-core V4
 * (spring_set_precision BF16 / BF16x3, two-atom cells) the work is proportional to the selected
 * branches; the FP64 path computes every branch.  rate(Ndof,n_q0,n_temps) receives the selected
 * rates and zero elsewhere; the resident LW_Allq0 is not touched.  Used by the surrogate-screened
 * path to spend exact evaluation on the modes it ranks first. */
int spring_linewidth4_modes(spring_ctx* ctx, int i0_first, int n_q0, double sigma, const int* s0_mask, double* rate);

/* ---- LineWidth.x path mode ------------------------------------------- */
/* q_points_highsymm, src/LineWidth/Src/CreateMesh_mod.f90:85-172: path points
 * from q_high_sym(4,n_nodes) (fractional node, points on the segment ending at
 * it).  *n_rows = points written (the reference allocates sum(q_high_sym(4,:))
 * rows and fills this many); qpoints(3,*) Cartesian, dist(*) and
 * zero_centered(*) (1 when the segment uses the zero-centred q1 mesh) may be
 * NULL (then only *n_rows is returned). */
int spring_path_qpoints(spring_ctx* ctx, int n_nodes, const double* q_high_sym, int* n_rows, double* qpoints,
                        double* dist, int* zero_centered);

/* Linewidth at off-grid q0 points, the q0 loop of src/LineWidth/Src/main.f90:297-389:
 * ScatterProbAllq1 (Linewidth_m.f90:48-231: q2 = G - q0 - q1 found inside the
 * zone in fractional coordinates, phonons of every q2 on the device) and
 *   SPRING_DELTA_TETRA: CalculateLwTetrahedron (Linewidth_m.f90:326-417), or
 *   SPRING_DELTA_GAUSS: CalculateLinewidth (:234-323, branch start reset per q1).
 * q0(3,n_q0) Cartesian, zero_centered(n_q0) from spring_path_qpoints.  Needs
 * FC2, FC3, a zero-centred mesh and its grid phonons; non-zero-centred segments
 * take their q1 vectors from the [0, N) mesh and the phonons of the same grid
 * points.  lw(Ndof,n_q0,n_temps) and omega_q0(Ndof,n_q0) are optional outputs;
 * the resident LW_Allq0 is not touched. */
int spring_linewidth_path(spring_ctx* ctx, int n_q0, const double* q0, const int* zero_centered, int delta_mode,
                          double sigma, double* lw, double* omega_q0);

/* Arithmetic of the 3- and 4-phonon matrix elements in the Gaussian rates
 * (spring_linewidth3 / spring_linewidth4 / spring_linewidth4_modes with SPRING_DELTA_GAUSS,
 * two-atom cells; spring_linewidth4 over every branch): SPRING_FP64 (default), SPRING_BF16 or
 * SPRING_BF16X3, the contractions on the tensor cores with FP64 frequencies, occupations, delta
 * weights and sums.  No counterpart in the reference, which is FP64 throughout.  Other cells and
 * the tetrahedron path stay FP64. */
int spring_set_precision(spring_ctx* ctx, int precision);

/* ---- surrogate network of the screened four-phonon path -------------- */
/* No counterpart in the reference, which evaluates every four-phonon rate
 * exactly.  A 5 -> 128 -> 128 -> 128 -> 1 network (SiLU) that maps per-mode
 * harmonic features to the log four-phonon rate, trained and evaluated on the
 * device; its error is measured against the exact spring_linewidth4.
 * X(SPRING_MLP_INPUTS, n) features (standardised by the caller), y(n) targets.
 * Parameters: one FP32 vector of SPRING_MLP_PARAMS values, W1 (128x5 row-major),
 * b1, W2 (128x128), b2, W3, b3, W4 (1x128), b4. */
#define SPRING_MLP_INPUTS 5
#define SPRING_MLP_PARAMS 33921
int spring_mlp_init(spring_ctx* ctx, unsigned long long seed);
int spring_mlp_set_params(spring_ctx* ctx, const float* params);
int spring_mlp_get_params(spring_ctx* ctx, float* params);
/* Mean-squared-error loss and its gradient (SPRING_MLP_PARAMS) over all n rows. */
int spring_mlp_loss_grad(spring_ctx* ctx, int n, const float* X, const float* y, float* loss, float* grad);
/* Adam (beta 0.9/0.999) over `epochs` shuffled passes in minibatches of `batch`
 * rows (a trailing partial batch is skipped); epoch_loss(epochs) optional. */
int spring_mlp_train(spring_ctx* ctx, int n, const float* X, const float* y, int epochs, int batch, float lr,
                     unsigned long long seed, float* epoch_loss);
/* y(n) = network(X); bf16 != 0 rounds weights and activations to BF16. */
int spring_mlp_predict(spring_ctx* ctx, int n, const float* X, float* y, int bf16);

/* Zero / read / replace the resident LW_Allq0(Ndof,Nq0,n_temps). */
int spring_reset_linewidths(spring_ctx* ctx);
int spring_get_linewidths(spring_ctx* ctx, double* lw_all);
int spring_set_linewidths(spring_ctx* ctx, const double* lw_all);

/* ---- thermal conductivity --------------------------------------------- */
/* RTA kappa per temperature, kappa(9,n_temps) in kron_prod order.
 *   symm = 1: GrVelKronProdSymm + kappa_noIter_symm (VelocityKronProd_symm.f90:34-91,
 *             ThermalConductivity.f90:167-292); Rxyz(3,3,nsym) Cartesian rotations.
 *   symm = 0: kappa_noIter over the full grid (ThermalConductivity.f90:36-164).
 * s_range(2): branch window (min/max of Polarization3rd/4th first column) or NULL.
 * mode_k(9,Ndof,n_temps) optional (ModeResolvedKappa). Uses the resident LW_Allq0. */
int spring_kappa_rta(spring_ctx* ctx, int symm, int nsym, const double* Rxyz, const int* s_range, double* kappa,
                     double* mode_k);

/* Iterative (non-RTA) kappa of kappa_iter.x (src/Kappa/Src_iterative/main.f90:219-361):
 * time-reversal irreducible set, tetrahedron 1/tau and F0 (CreateFzero), then
 * F <- F0 + tau * sum(...) until max|kappa_new - kappa_old| < eps_k or more than
 * max_iter iterations (MAX_ITER = 1000 in the reference), for every temperature.
 * Uses the grid phonons and FC3.  kappa(9,n_temps), kappa_rta(9,n_temps) (iteration
 * 0) and iters(n_temps) are outputs (NULL allowed). */
int spring_kappa_iter(spring_ctx* ctx, double eps_k, int max_iter, double* kappa, double* kappa_rta, int* iters);

/* The same iteration with Gaussian delta weights of width sigma (THz) in place of the
 * tetrahedra: both channels of TetrahedronIterPlus / TetrahedronIterMinus
 * (src/Kappa/Src_iterative/Quasi_momentum_consrv.f90:701-1208) with d(w0 - M) a
 * Gaussian, as kappa.x's Gaussian linewidths are to its tetrahedron ones.  The scattering
 * operator (one entry per pair and mode triple inside the exp(-40) window) is built once
 * on the device, sorted by row and kept until sigma, FC3 or the phonons change; every
 * iteration is then one pass over it.  Two-atom cells with 7-atom FC3 clusters.
 * On a context set to SPRING_BF16 / SPRING_BF16X3 the operator entries come
 * from the tensor-core V3 pass (same window and cuts; |Phi|^2 in compensated
 * BF16), the iterations stay FP64.
 * stats(2) optional: number of operator entries, number of enumerated pairs. */
int spring_kappa_iter_gauss(spring_ctx* ctx, double sigma, double eps_k, int max_iter, double* kappa,
                            double* kappa_rta, int* iters, double* stats);

/* ---- batched linewidths (several workloads, one persistent launch) ------ */
/* A batch holds Gaussian three-phonon linewidth requests on several contexts
 * (different cells, meshes and temperature sets, on one device) and runs them
 * as one persistent FP64 kernel over all their (pair, s0-block) work items,
 * heaviest workloads first, captured with its zero-fills and the LW_Allq0
 * updates in one CUDA graph that later runs replay.  Each request has the
 * meaning of spring_linewidth3(ctx, i0_first, n_q0, SPRING_DELTA_GAUSS, sigma,
 * pol3, ...) on its context (the q0 loop body of main.f90:552-715 for many
 * inputs at once); no counterpart in the reference, which runs one input per
 * process.  Requests on one context must not overlap in q0.  A request on a
 * two-atom context set to SPRING_BF16 / SPRING_BF16X3 runs through the
 * tensor-core pass of spring_linewidth3 (same kernel, same results) right
 * after the graph, inside the same spring_batch_run; path requests
 * (spring_batch_add_path) are launched inside the graph. */
typedef struct spring_batch spring_batch;
int spring_batch_create(spring_batch** batch);
int spring_batch_destroy(spring_batch* batch);
const char* spring_batch_last_error(const spring_batch* batch);
/* Add a request; returns its index (0-based) in *index (may be NULL). */
int spring_batch_add_linewidth3(spring_batch* batch, spring_ctx* ctx, int i0_first, int n_q0, double sigma,
                                const int* pol3, int* index);
/* Launch configuration of the persistent kernel (288 threads per CTA):
 * config[0] 1 = two-atom cells (7-atom FC3 clusters, <= 9 temperatures) run as
 * groups of 8 pairs in the specialised layout, 0 = every cell as (pair, s0
 * block) items of the any-cell layout; config[1] CTAs per SM (0 = as many as
 * fit); config[2] s0 block for cells with Ndof > 12 (0 = 6, or 6, 12, 24);
 * config[3] work items taken per scheduler step.  Default {1, 0, 0, 1}. */
int spring_batch_set_config(spring_batch* batch, const int* config);
int spring_batch_get_config(const spring_batch* batch, int* config);
/* Autotuner: time the batch under candidate configurations (coordinate search
 * over the four parameters, each run timed with CUDA events; LW_Allq0 is not
 * touched) and keep the fastest.  The result is cached for the process by the
 * batch's shape (cells, meshes, temperatures, pair counts), so a later batch
 * of the same shape starts tuned.  best_ms and n_tried may be NULL. */
int spring_batch_tune(spring_batch* batch, int* config, double* best_ms, int* n_tried);
/* Run every request (accumulating into each context's LW_Allq0, as
 * spring_linewidth3 does); the first run captures the CUDA graph. */
int spring_batch_run(spring_batch* batch);
/* Results of request `index` of the last run: lw(Ndof,n_q0,n_temps) and
 * P3_q0(Ndof,n_q0) of its context (either may be NULL); device time of the last
 * run in *ms (may be NULL). */
int spring_batch_result(spring_batch* batch, int index, double* lw, double* p3_q0, double* ms);
/* Gaussian linewidths at n_path off-grid points of a context, as
 * spring_linewidth_path(ctx, n_path, q_path, zero_centered, SPRING_DELTA_GAUSS,
 * sigma, ...) computes them (LineWidth.x path mode, src/LineWidth/Src/main.f90:293-379),
 * queued in the batch's graph after the persistent kernel.  Its buffers are
 * allocated at the first spring_batch_run; add a linewidth request first (it
 * binds the batch's device).  Returns its index among the path requests. */
int spring_batch_add_path(spring_batch* batch, spring_ctx* ctx, int n_path, const double* q_path,
                          const int* zero_centered, double sigma, int* index);
/* lw(Ndof,n_path,n_temps) and omega(Ndof,n_path) of path request `index` after the last run
 * (either may be NULL). */
int spring_batch_path_result(spring_batch* batch, int index, double* lw, double* omega);

/* ---- options ----------------------------------------------------------- */
/* SPRING_OPT_GENERIC_V3 = 1: always use the any-cell V3 kernel (default 0 picks the
 * two-atom specialisation when the cell fits it; both give the same W). */
#define SPRING_OPT_GENERIC_V3 1
/* SPRING_OPT_WAIT_POLLS = 2: poll limit of each wait of one warp on another inside the
 * tensor-core kernels (value >= 0; a negative value restores the default, 2^26).  When a wait
 * runs out, the kernel drains the copies and MMAs it issued, releases its shared and tensor
 * memory and returns; the call fails with SPRING_ERR_TIMEOUT.  For testing callers' handling
 * of that status: 0 makes every such wait run out at once. */
#define SPRING_OPT_WAIT_POLLS 2
/* SPRING_OPT_FP64_PRESCREEN = 3: value 1 makes the FP64 Gaussian 3-phonon linewidth of two-atom
 * cells (k_v3s) skip the pairs with no mode triple inside the window where a delta weight exceeds
 * exp(-40) of its peak (the tensor-core path's pre-screen; the linewidths change below 1e-13
 * relative); 0 (default) evaluates every pair. */
#define SPRING_OPT_FP64_PRESCREEN 3
int spring_set_option(spring_ctx* ctx, int option, int value);

/* ---- diagnostics ------------------------------------------------------- */
/* Record CUDA events around every kernel launch (on = 1) or stop (on = 0);
 * turning it on clears earlier records. */
int spring_set_profiling(spring_ctx* ctx, int on);
/* Device time (ms) and launch count of the recorded launches whose kernel
 * name starts with `prefix` (e.g. "k_v3"); synchronizes the stream. */
int spring_kernel_time(spring_ctx* ctx, const char* prefix, double* ms, long long* launches);
/* Binary architecture of this library's kernels as the runtime loaded them on `device`
 * (cudaFuncGetAttributes binaryVersion: 100 for sm_100a).  No reference counterpart. */
int spring_binary_version(int device, int* version);
/* Pairs and 16-pair tiles of the last tensor-core linewidth pass (the pairs with a mode
 * triple inside the delta window); 0 and 0 before one ran.  No reference counterpart. */
int spring_tc_stats(const spring_ctx* ctx, int* n_tiles, int* n_pairs);

/* Make the n-th (1-based) subsequent device allocation (kind 0), host<->device
 * copy (kind 1) or kernel launch (kind 2) report failure without performing
 * it; n = 0 disarms.  For testing callers' error paths. */
int spring_debug_inject_fault(spring_ctx* ctx, int kind, int n);

#ifdef __cplusplus
}
#endif
#endif /* SPRING_GPU_H */
