// libspring_host.so: the reference's FC input files and result files (see include/spring_host.h).
#include <cstring>
#include <string>
#include <vector>

#include "../../include/spring_host.h"
#include "ewald.hpp"
#include "h5lite.hpp"

namespace {

thread_local std::string g_err;

int fail(const std::string& m) {
    g_err = m;
    return 1;
}

std::string mu_name(int order, int mu) {  // 'FC3_mu'//trim(adjustl(I2 of mu)), hdf5_wrap_mod.f90:186
    return std::string(order == 3 ? "FC3_mu" : "FC4_mu") + std::to_string(mu);
}

const h5lite::Dataset* find(const h5lite::Group& g, const std::string& path) {
    const size_t slash = path.find('/');
    if (slash == std::string::npos) {
        auto it = g.datasets.find(path);
        return it == g.datasets.end() ? nullptr : &it->second;
    }
    auto it = g.groups.find(path.substr(0, slash));
    return it == g.groups.end() ? nullptr : find(*it->second, path.substr(slash + 1));
}

}  // namespace

extern "C" {

const char* spring_host_last_error(void) { return g_err.c_str(); }

int spring_h5_write_fc(const char* path, int order, int nb, int na, const int* atm_num, const int* atm_indx,
                       const double* fc) {
    if (!path || !atm_num || !atm_indx || !fc || nb < 1 || na < 1 || order < 2 || order > 4)
        return fail("spring_h5_write_fc: bad arguments");
    h5lite::Group root;
    root.datasets["NumAtoms"] = h5lite::make_i32(atm_num, {(uint64_t)nb});
    root.datasets["atm_Indx"] = h5lite::make_i32(atm_indx, {4, (uint64_t)na, (uint64_t)nb});
    if (order == 2) {
        root.datasets["FC2"] = h5lite::make_f64(fc, {1, 3, 3, (uint64_t)na, (uint64_t)nb});
    } else {
        h5lite::Group& g = root.group(order == 3 ? "FC3rd" : "FC4th");
        const size_t per = order == 3 ? (size_t)27 * na * na : (size_t)81 * na * na * na;
        for (int mu = 0; mu < nb; ++mu) {
            std::vector<uint64_t> fd = order == 3 ? std::vector<uint64_t>{3, 3, 3, (uint64_t)na, (uint64_t)na}
                                                  : std::vector<uint64_t>{3, 3, 3, 3, (uint64_t)na, (uint64_t)na, (uint64_t)na};
            g.datasets[mu_name(order, mu + 1)] = h5lite::make_f64(fc + per * mu, fd);
        }
    }
    const std::string e = h5lite::write_file(path, root);
    return e.empty() ? 0 : fail(e);
}

int spring_h5_fc_dims(const char* path, int order, int* nb, int* na) {
    if (!path || !nb || !na) return fail("spring_h5_fc_dims: bad arguments");
    h5lite::Group root;
    std::string e = h5lite::read_file(path, root);
    if (!e.empty()) return fail(e);
    const h5lite::Dataset* num = find(root, "NumAtoms");
    if (!num || num->type != h5lite::Type::I32 || num->dims.size() != 1) return fail(std::string(path) + ": no NumAtoms");
    *nb = (int)num->dims[0];
    const int32_t* v = reinterpret_cast<const int32_t*>(num->data.data());
    int m = 0;
    for (int i = 0; i < *nb; ++i) m = std::max(m, (int)v[i]);
    const h5lite::Dataset* idx = find(root, "atm_Indx");
    if (!idx || idx->dims.size() != 3) return fail(std::string(path) + ": no atm_Indx(4,na,nb)");
    // FC2's cluster extent is the second dimension of atm_Indx (the reference allocates from it)
    *na = order == 2 ? (int)idx->dims[1] : m;
    (void)order;
    return 0;
}

int spring_h5_read_fc(const char* path, int order, int nb, int na, int* atm_num, int* atm_indx, double* fc) {
    if (!path || !atm_num || !atm_indx || !fc || nb < 1 || na < 1 || order < 2 || order > 4)
        return fail("spring_h5_read_fc: bad arguments");
    h5lite::Group root;
    std::string e = h5lite::read_file(path, root);
    if (!e.empty()) return fail(e);
    const h5lite::Dataset* num = find(root, "NumAtoms");
    const h5lite::Dataset* idx = find(root, "atm_Indx");
    if (!num || !idx || num->type != h5lite::Type::I32 || idx->type != h5lite::Type::I32)
        return fail(std::string(path) + ": NumAtoms / atm_Indx missing or not integers");
    if ((int)num->count() != nb) return fail(std::string(path) + ": NumAtoms has another size");
    std::memcpy(atm_num, num->data.data(), sizeof(int) * nb);
    // atm_Indx(4, na_file, nb) into atm_indx(4, na, nb)
    const std::vector<uint64_t> fi = h5lite::fortran_dims(*idx);
    if (fi.size() != 3 || fi[0] != 4 || (int)fi[2] != nb)
        return fail(std::string(path) + ": atm_Indx has an unexpected shape");
    std::memset(atm_indx, 0, sizeof(int) * 4 * na * nb);
    const int32_t* iv = reinterpret_cast<const int32_t*>(idx->data.data());
    const int naf = (int)fi[1];
    for (int mu = 0; mu < nb; ++mu)
        for (int n = 0; n < std::min(na, naf); ++n)
            for (int k = 0; k < 4; ++k) atm_indx[4 * (n + (size_t)na * mu) + k] = iv[4 * (n + (size_t)naf * mu) + k];
    const int blk = order == 2 ? 9 : (order == 3 ? 27 : 81);
    const int nslot = order == 2 ? 1 : (order == 3 ? 2 : 3);
    size_t per = blk;
    for (int s = 0; s < nslot; ++s) per *= (size_t)na;
    std::memset(fc, 0, sizeof(double) * per * nb);
    if (order == 2) {
        const h5lite::Dataset* d = find(root, "FC2");
        if (!d || d->type != h5lite::Type::F64) return fail(std::string(path) + ": FC2 missing or not double");
        const std::vector<uint64_t> fd = h5lite::fortran_dims(*d);
        if (fd.size() != 5 || fd[0] != 1 || fd[1] != 3 || fd[2] != 3 || (int)fd[4] != nb || (int)fd[3] > na)
            return fail(std::string(path) + ": FC2 has an unexpected shape");
        const double* v = reinterpret_cast<const double*>(d->data.data());
        for (int mu = 0; mu < nb; ++mu)
            for (int n = 0; n < (int)fd[3]; ++n)
                std::memcpy(fc + 9 * (n + (size_t)na * mu), v + 9 * (n + fd[3] * mu), sizeof(double) * 9);
        return 0;
    }
    for (int mu = 0; mu < nb; ++mu) {
        const std::string name = std::string(order == 3 ? "FC3rd/" : "FC4th/") + mu_name(order, mu + 1);
        const h5lite::Dataset* d = find(root, name);
        if (!d || d->type != h5lite::Type::F64) return fail(std::string(path) + ": " + name + " missing or not double");
        const std::vector<uint64_t> fd = h5lite::fortran_dims(*d);
        if ((int)fd.size() != (order == 3 ? 5 : 7)) return fail(std::string(path) + ": " + name + " has an unexpected rank");
        const int nf = (int)fd[order == 3 ? 3 : 4];
        if (nf > na) return fail(std::string(path) + ": " + name + " is larger than NumAtoms allows");
        const double* v = reinterpret_cast<const double*>(d->data.data());
        double* out = fc + per * mu;
        if (order == 3) {
            for (int n2 = 0; n2 < nf; ++n2)
                for (int n1 = 0; n1 < nf; ++n1)  // the two slot dimensions, first one fastest
                    std::memcpy(out + 27 * (n1 + (size_t)na * n2), v + 27 * (n1 + (size_t)nf * n2), sizeof(double) * 27);
        } else {
            for (int n3 = 0; n3 < nf; ++n3)
                for (int n2 = 0; n2 < nf; ++n2)
                    for (int n1 = 0; n1 < nf; ++n1)
                        std::memcpy(out + 81 * (n1 + (size_t)na * (n2 + (size_t)na * n3)),
                                    v + 81 * (n1 + (size_t)nf * (n2 + (size_t)nf * n3)), sizeof(double) * 81);
        }
    }
    return 0;
}

int spring_h5_write_kappa(const char* path, const double* kappa, int ndof, int nq0, const double* linewidth,
                          const double* phase_space, const double* mode_k, const double* scatter_pd) {
    if (!path || !kappa || !linewidth || !phase_space || ndof < 1 || nq0 < 1) return fail("spring_h5_write_kappa: bad arguments");
    h5lite::Group root;
    root.datasets["ThermalConductivityTensor"] = h5lite::make_f64(kappa, {9});
    root.datasets["LineWidth"] = h5lite::make_f64(linewidth, {(uint64_t)(2 * ndof), (uint64_t)nq0});
    root.datasets["PhaseSpace3rd"] = h5lite::make_f64(phase_space, {(uint64_t)(2 * ndof), (uint64_t)nq0});
    if (mode_k) root.datasets["ModeResolvedKappa"] = h5lite::make_f64(mode_k, {9, (uint64_t)ndof});
    if (scatter_pd) root.datasets["Scatter_pd"] = h5lite::make_f64(scatter_pd, {(uint64_t)(2 * ndof), (uint64_t)nq0});
    const std::string e = h5lite::write_file(path, root);
    return e.empty() ? 0 : fail(e);
}

int spring_h5_write_restart(const char* path, int ndof, int nq0, int i0, int complete, const double* lw) {
    if (!path || !lw || ndof < 1 || nq0 < 1) return fail("spring_h5_write_restart: bad arguments");
    h5lite::Group root;
    const int32_t prog[2] = {i0, complete};
    root.datasets["progress"] = h5lite::make_i32(prog, {2});
    root.datasets["LW_data"] = h5lite::make_f64(lw, {(uint64_t)ndof, (uint64_t)nq0});
    const std::string e = h5lite::write_file(path, root);
    return e.empty() ? 0 : fail(e);
}

int spring_h5_read_restart(const char* path, int ndof, int nq0, int* progress, double* lw) {
    if (!path || !progress || !lw) return fail("spring_h5_read_restart: bad arguments");
    h5lite::Group root;
    std::string e = h5lite::read_file(path, root);
    if (!e.empty()) return fail(e);
    const h5lite::Dataset* p = find(root, "progress");
    const h5lite::Dataset* d = find(root, "LW_data");
    if (!p || p->type != h5lite::Type::I32 || p->count() != 2) return fail(std::string(path) + ": no progress(2)");
    if (!d || d->type != h5lite::Type::F64) return fail(std::string(path) + ": no LW_data");
    const std::vector<uint64_t> fd = h5lite::fortran_dims(*d);
    if (fd.size() != 2 || (int)fd[0] != ndof || (int)fd[1] != nq0)
        return fail(std::string(path) + ": LW_data is not (Ndof, Nq0) of this run");
    std::memcpy(progress, p->data.data(), 2 * sizeof(int));
    std::memcpy(lw, d->data.data(), d->data.size());
    return 0;
}

int spring_h5_read_f64(const char* path, const char* name, int* rank, long long* fdims, double* out, long long cap) {
    if (!path || !name || !rank || !fdims) return fail("spring_h5_read_f64: bad arguments");
    h5lite::Group root;
    std::string e = h5lite::read_file(path, root);
    if (!e.empty()) return fail(e);
    const h5lite::Dataset* d = find(root, name);
    if (!d) return fail(std::string(path) + ": no dataset " + name);
    if (d->type != h5lite::Type::F64) return fail(std::string(path) + ": " + name + " is not double");
    const std::vector<uint64_t> fd = h5lite::fortran_dims(*d);
    if (fd.size() > 8) return fail("rank above 8");
    *rank = (int)fd.size();
    for (size_t i = 0; i < fd.size(); ++i) fdims[i] = (long long)fd[i];
    if (out) {
        if ((long long)d->count() > cap) return fail("output buffer too small");
        std::memcpy(out, d->data.data(), d->data.size());
    }
    return 0;
}

int spring_ewald_setup(const double* latvec, int nb, const double* atm_pos, const double* dielec, const double* born_z,
                       int decide, double prec_ew, double lmb, const int* gmesh, const int* rmesh, const int* sup_cell,
                       double* lmb_out, int* gmesh_out, int* counts, double* cc_out, double* hz_out, long long hz_cap) {
    if (!latvec || !atm_pos || !dielec || !born_z || !rmesh || !sup_cell) return fail("spring_ewald_setup: bad arguments");
    spring_ewald::Setup S;
    std::string err;
    if (spring_ewald::setup(latvec, nb, atm_pos, dielec, born_z, decide, prec_ew, lmb, gmesh, rmesh, sup_cell, S, err))
        return fail(err);
    if (lmb_out) *lmb_out = S.lmb;
    if (gmesh_out)
        for (int k = 0; k < 3; ++k) gmesh_out[k] = S.gmesh[k];
    if (counts) {
        counts[0] = S.nr();
        counts[1] = S.ng();
    }
    if (cc_out) std::memcpy(cc_out, S.cc.data(), sizeof(double) * S.cc.size());
    if (hz_out) {
        if ((long long)S.hz.size() > hz_cap) return fail("spring_ewald_setup: hz buffer too small");
        std::memcpy(hz_out, S.hz.data(), sizeof(double) * S.hz.size());
    }
    return 0;
}

}  // extern "C"
