/*
 * spring_host.h — host-side C ABI of libspring_host.so: the file formats around the hot path.
 *
 * The reference reads its force constants from HDF5 files and writes its results to an HDF5 file
 * and a text file (src/Kappa/Src/hdf5_wrap_mod.f90, src/Kappa/Src/Helper_m.f90:597-667).  These
 * entry points read and write the same files without the HDF5 library (h5lite), so that the
 * command-line driver spring_kappa and the tests can use the reference's inputs and outputs.
 * Arrays are the reference's Fortran arrays (column-major), shapes written in Fortran order.
 * Every call returns 0 on success; spring_host_last_error() gives the message of the last failure.
 */
#ifndef SPRING_HOST_H
#define SPRING_HOST_H

#ifdef __cplusplus
extern "C" {
#endif

const char* spring_host_last_error(void);

/* Write an FC file of `order` (2, 3 or 4) in the reference's layout (r2ndFC / r3rdFC / r4thFC,
 * hdf5_wrap_mod.f90:40-337): NumAtoms(nb), atm_Indx(4,na,nb) and FC2(1,3,3,na,nb), or groups
 * FC3rd/FC3_mu<k> = fc(3,3,3,na,na,k), FC4th/FC4_mu<k> = fc(3,3,3,3,na,na,na,k). */
int spring_h5_write_fc(const char* path, int order, int nb, int na, const int* atm_num, const int* atm_indx,
                       const double* fc);
/* Sizes of an FC file: *nb basis atoms, *na = maxval(NumAtoms) (the cluster extent). */
int spring_h5_fc_dims(const char* path, int order, int* nb, int* na);
/* Read an FC file into caller arrays sized by spring_h5_fc_dims (zero beyond each dataset). */
int spring_h5_read_fc(const char* path, int order, int nb, int na, int* atm_num, int* atm_indx, double* fc);

/* Write kappa_<prefix><T>K.h5 like kappa.x (main.f90:775-798, w1dh5_no_grp / w2dh5_no_grp_type2 /
 * w2dh5_no_grp, hdf5_wrap_mod.f90:650-766): ThermalConductivityTensor(9) = kappa, LineWidth and
 * PhaseSpace3rd (2 Ndof, nq0) = omega in rows 1..Ndof and the value in Ndof+1..2 Ndof, and
 * ModeResolvedKappa(9, Ndof) when mode_k is not NULL, Scatter_pd (2 Ndof, nq0) (the point-defect
 * rates with omega alongside, main.f90:778) when scatter_pd is not NULL. */
int spring_h5_write_kappa(const char* path, const double* kappa, int ndof, int nq0, const double* linewidth,
                          const double* phase_space, const double* mode_k, const double* scatter_pd);

/* The linewidth restart file of kappa.x (w_RestartLW / r_RestartLW, hdf5_wrap_mod.f90:340-401 and
 * :562-647; Restart_<prefix>/<prefix><T>K_LW_Restart.h5): progress(2) = (last irreducible point
 * done, 1 when it completed) and LW_data(Ndof, Nq0). */
int spring_h5_write_restart(const char* path, int ndof, int nq0, int i0, int complete, const double* lw);
int spring_h5_read_restart(const char* path, int ndof, int nq0, int* progress, double* lw);

/* One double dataset at `name` ("a/b" for a dataset in a group): *rank and fdims (Fortran order,
 * up to 8); the data go to out when out != NULL and cap (elements) is large enough. */
int spring_h5_read_f64(const char* path, const char* name, int* rank, long long* fdims, double* out, long long cap);

/* The host part of the dipole-dipole term (the same code the device library runs in
 * spring_set_dipole): Lmb and Gmesh (DecideEwaldParameters when decide != 0), counts = (number of R
 * points, number of G points), cc(2, 9 Nb^2) = -CombineZStar(CConst) - CSumq0 on the diagonal
 * blocks (complex, C(beta, alpha, nu, mu) order), hz(9 Nb^2, NR) the Born-charge-folded real-space
 * terms.  Any output may be NULL.  Arguments as spring_set_dipole plus latvec(3,3). */
int spring_ewald_setup(const double* latvec, int nb, const double* atm_pos, const double* dielec, const double* born_z,
                       int decide, double prec_ew, double lmb, const int* gmesh, const int* rmesh, const int* sup_cell,
                       double* lmb_out, int* gmesh_out, int* counts, double* cc_out, double* hz_out, long long hz_cap);

#ifdef __cplusplus
}
#endif
#endif
