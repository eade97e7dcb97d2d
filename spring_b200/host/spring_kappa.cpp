// spring_kappa: the command-line driver of kappa.x (src/Kappa/Src/main.f90) on the B200 library.
//
//   spring_kappa -inp input.nml -T 300 [-omegacut w] [-Mode_resolved_k T|F] [-Symm T|F]
//                [-precision fp64|bf16|bf16x3] [-delta tetra|gauss] [-dry-run]
//
// Same command line (get_command_line, src/Kappa/Src/parse_cmd_line.f90:37-275), namelists
// (&FCInfo, &CrystalInfo, &AtmInfo: unit_mod.f90:64-209; &AnhInfo: Helper_m.f90:37-132), input
// files FC2nd_/FC3rd_/FC4th_<prefix><T>K_F.h5 and outputs as kappa.x: kappa_<prefix><T>K.h5 with
// ThermalConductivityTensor(9), LineWidth and PhaseSpace3rd (2 Ndof x Nq0: omega, then the value;
// main.f90:775-777) and ModeResolvedKappa(9, Ndof) (:798), and linewidth_IBZ_<prefix><T>K.txt
// (WriteAsciiOutFile, Helper_m.f90:597-667, format Ndof-1 (G20.12,'  '), G20.12).  Every q0 is
// computed by the library in one call (the q0 loop of main.f90:552-715): tetrahedron 3-phonon
// linewidths (the scheme kappa.x ships; -delta gauss uses Sigma), isotope scattering when isotope
// is set, four-phonon rates when FourPhonon is set, RTA kappa (symmetrised by default); with
// WriteRestart / ReadRestart the linewidth restart file (main.f90:502-545) is rewritten after every
// block of points and read back to skip the points already done.  The point
// group comes from the lattice and basis (the rotations spg_get_symmetry gives for a primitive
// cell); the phonons from the device eigensolver.  Extensions: -precision selects the tensor-core
// arithmetic of the Gaussian V3/V4; -dry-run reads and checks every input and prints them as JSON
// without a GPU.
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/spring_gpu.h"
#include "../../include/spring_host.h"
#include "namelist.hpp"

namespace {

[[noreturn]] void die(const std::string& m) {
    std::fprintf(stderr, "spring_kappa: %s\n", m.c_str());
    std::exit(1);
}

void check(const std::string& e) {
    if (!e.empty()) die(e);
}

bool to_bool(const std::string& s) {
    return !s.empty() && (s[0] == 'T' || s[0] == 't' || (s[0] == '.' && s.size() > 1 && (s[1] == 'T' || s[1] == 't')));
}

// Fortran G20.12 of one value: F(w-4).(d-k) and four blanks where 0.1 <= |x| < 10^d (k = digits
// before the point after rounding to d significant digits), else E20.12 (0.ddd...E+xx).
std::string g20(double x) {
    const int w = 20, d = 12;
    char buf[64];
    if (x == 0.0) {
        std::snprintf(buf, sizeof buf, "%*.*f    ", w - 4, d - 1, 0.0);
        return buf;
    }
    const double ax = std::fabs(x);
    std::snprintf(buf, sizeof buf, "%.*e", d - 1, ax);  // d significant digits
    const int e10 = std::atoi(std::strchr(buf, 'e') + 1);
    if (ax >= 0.1 - 0.5e-13 && e10 + 1 <= d) {
        const int k = std::max(e10 + 1, 0);
        std::snprintf(buf, sizeof buf, "%*.*f    ", w - 4, d - k, x);
        return buf;
    }
    std::string digits;
    for (const char* p = buf; *p && *p != 'e'; ++p)
        if (*p >= '0' && *p <= '9') digits.push_back(*p);
    const int ex = e10 + 1;
    char eb[16];
    if (std::abs(ex) <= 99) std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    const std::string s = std::string(x < 0 ? "-" : "") + "0." + digits + eb;
    return std::string(std::max(0, w - (int)s.size()), ' ') + s;
}

// Point-group rotations W (fractional, x' = W x; entries -1, 0, 1) that keep the metric and map
// the basis onto itself (same type) up to one translation: what spg_get_symmetry returns as
// rotations for a primitive cell (src/Kappa/Src/Symmetry_m.f90:84).  Row-major W.
std::vector<int> point_group(const std::vector<double>& lat /* latvec(3,3), columns */, const std::vector<double>& pos,
                             const std::vector<int>& typ, int nb, double symprec) {
    double Lm[3][3], M[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) Lm[r][c] = lat[r + 3 * c];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            M[i][j] = 0.0;
            for (int r = 0; r < 3; ++r) M[i][j] += Lm[r][i] * Lm[r][j];
        }
    double scale = 0.0;
    for (int i = 0; i < 3; ++i) scale = std::max(scale, M[i][i]);
    std::vector<int> out;
    int W[9];
    for (int code = 0; code < 19683; ++code) {
        int c = code;
        for (int k = 0; k < 9; ++k) {
            W[k] = c % 3 - 1;
            c /= 3;
        }
        const int det = W[0] * (W[4] * W[8] - W[5] * W[7]) - W[1] * (W[3] * W[8] - W[5] * W[6]) +
                        W[2] * (W[3] * W[7] - W[4] * W[6]);
        if (det != 1 && det != -1) continue;
        bool metric = true;  // W^T M W == M
        for (int i = 0; i < 3 && metric; ++i)
            for (int j = 0; j < 3 && metric; ++j) {
                double s = 0.0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) s += W[3 * a + i] * M[a][b] * W[3 * b + j];
                metric = std::fabs(s - M[i][j]) <= 1e-6 * scale;
            }
        if (!metric) continue;
        auto apply = [&](int i, double* y) {
            for (int r = 0; r < 3; ++r)
                y[r] = W[3 * r] * pos[3 * i] + W[3 * r + 1] * pos[3 * i + 1] + W[3 * r + 2] * pos[3 * i + 2];
        };
        auto close = [&](const double* a, const double* b) {
            double d[3], cart[3] = {0, 0, 0};
            for (int r = 0; r < 3; ++r) d[r] = a[r] - b[r] - std::round(a[r] - b[r]);
            for (int r = 0; r < 3; ++r)
                for (int k = 0; k < 3; ++k) cart[r] += Lm[r][k] * d[k];
            return std::sqrt(cart[0] * cart[0] + cart[1] * cart[1] + cart[2] * cart[2]) <= symprec;
        };
        double y0[3];
        apply(0, y0);
        bool found = false;
        for (int j = 0; j < nb && !found; ++j) {
            if (typ[j] != typ[0]) continue;
            double t[3];
            for (int r = 0; r < 3; ++r) t[r] = pos[3 * j + r] - y0[r];
            bool all = true;
            for (int i = 0; i < nb && all; ++i) {
                double y[3];
                apply(i, y);
                for (int r = 0; r < 3; ++r) y[r] += t[r];
                bool hit = false;
                for (int k = 0; k < nb && !hit; ++k) hit = typ[k] == typ[i] && close(y, &pos[3 * k]);
                all = hit;
            }
            found = all;
        }
        if (found) out.insert(out.end(), W, W + 9);
    }
    return out;
}

std::string temp_char(double T) {  // write(Temp_char, '(F6.1)') T, trimmed
    char b[32];
    std::snprintf(b, sizeof b, "%6.1f", T);
    std::string s(b);
    return s.substr(s.find_first_not_of(' '));
}

struct Fc {
    int nb = 0, na = 0;
    std::vector<int> num, idx;
    std::vector<double> fc;
};

Fc read_fc(const std::string& path, int order) {
    Fc f;
    if (spring_h5_fc_dims(path.c_str(), order, &f.nb, &f.na)) die(spring_host_last_error());
    f.num.resize(f.nb);
    f.idx.resize((size_t)4 * f.na * f.nb);
    size_t per = order == 2 ? 9 : (order == 3 ? 27 : 81);
    for (int s = 0; s < (order == 2 ? 1 : order - 1); ++s) per *= (size_t)f.na;
    f.fc.resize(per * f.nb);
    if (spring_h5_read_fc(path.c_str(), order, f.nb, f.na, f.num.data(), f.idx.data(), f.fc.data()))
        die(spring_host_last_error());
    return f;
}

void gpu(spring_ctx* c, int rc) {
    if (rc) die(std::string("library: ") + spring_last_error(c));
}

}  // namespace

int main(int argc, char** argv) {
    std::string inp = "input.nml", precision = "fp64", delta = "tetra";
    double T = 300.0, freq_cut = 2.56789e-5;
    bool mode_k = false, symm = true, dry = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) die("missing value after " + a);
            return argv[++i];
        };
        if (a == "-inp") inp = val();
        else if (a == "-T") T = std::atof(val().c_str());
        else if (a == "-omegacut") freq_cut = std::atof(val().c_str());
        else if (a == "-Spectral_k") { if (to_bool(val())) die("-Spectral_k T is not supported by this driver"); }
        else if (a == "-Mode_resolved_k") mode_k = to_bool(val());
        else if (a == "-Symm") symm = to_bool(val());
        else if (a == "-precision") precision = val();
        else if (a == "-delta") delta = val();
        else if (a == "-dry-run") dry = true;
        else die("unknown argument " + a +
                 " (expected -inp FILE -T TEMP [-omegacut W] [-Mode_resolved_k T|F] [-Symm T|F] [-precision P] [-delta D])");
    }
    if (!(T > 0.0)) die("temperature must be positive");

    // ---- namelists
    std::map<std::string, nml::Group> groups;
    check(nml::parse_file(inp, groups));
    for (const char* gname : {"fcinfo", "crystalinfo", "atminfo"})
        if (!groups.count(gname)) die(std::string("namelist &") + gname + " missing in " + inp);
    const nml::Group &fci = groups["fcinfo"], &cri = groups["crystalinfo"], &ati = groups["atminfo"];
    nml::Group anh;
    if (groups.count("anhinfo")) anh = groups["anhinfo"];
    std::string prefix;
    check(nml::get(fci, "prefix", prefix));
    int nb = 2, ntyp = 1;
    check(nml::get(cri, "Nbasis", nb));
    check(nml::get(cri, "Ntyp", ntyp));
    if (nb < 1 || nb > 8 || ntyp < 1 || ntyp > nb) die("Nbasis must be 1..8 and Ntyp 1..Nbasis");
    std::vector<double> lat(9, 0.0), pos((size_t)3 * nb, 0.0), mass_unq(ntyp, 0.0);
    std::vector<int> typ(nb, 1);
    check(nml::get(cri, "Latvec", {3, 3}, lat));
    check(nml::get(ati, "atm_pos", {3, nb}, pos));
    check(nml::get(ati, "typ_indx", {nb}, typ));
    check(nml::get(ati, "mass", {ntyp}, mass_unq));
    std::vector<double> mass(nb);
    for (int i = 0; i < nb; ++i) {
        if (typ[i] < 1 || typ[i] > ntyp) die("typ_indx out of range");
        mass[i] = mass_unq[typ[i] - 1];
    }
    // &AnhInfo with the reference's defaults (ReadNmlKappa)
    std::vector<std::string> sel3(3, "D"), sel4(4, "D");
    double sigma = 5.1, symprec = 1e-7;
    std::vector<double> g2iso(nb, 0.0);
    std::vector<int> qmesh{7, 7, 7}, shift{0, 0, 0};
    int time_rev = 0;
    bool isotope = false, four = false, wrestart = false, rrestart = false;
    check(nml::get(anh, "SelectionRule3", {3}, sel3));
    check(nml::get(anh, "SelectionRule4", {4}, sel4));
    check(nml::get(anh, "Sigma", sigma));
    check(nml::get(anh, "symprec", symprec));
    check(nml::get(anh, "g2iso", {nb}, g2iso));
    check(nml::get(anh, "qmesh", {3}, qmesh));
    check(nml::get(anh, "shift", {3}, shift));
    check(nml::get(anh, "time_rev", time_rev));
    check(nml::get(anh, "isotope", isotope));
    check(nml::get(anh, "FourPhonon", four));
    check(nml::get(anh, "WriteRestart", wrestart));
    check(nml::get(anh, "ReadRestart", rrestart));
    const int ndof = 3 * nb;
    auto pol = [&](const std::vector<std::string>& sel) {  // PolarizationStrtEnd, Helper_m.f90:310-353
        std::vector<int> p;
        for (const auto& s : sel) {
            const char b = s.empty() ? 'D' : s[0];
            if (b == 'A' || b == 'a') p.insert(p.end(), {1, 3});
            else if (b == 'O' || b == 'o') p.insert(p.end(), {4, ndof});
            else p.insert(p.end(), {1, ndof});
        }
        return p;
    };
    const std::vector<int> pol3 = pol(sel3), pol4 = pol(sel4);
    // Dipole-dipole term: &FCInfo Force_dd, &CrystalInfo Sup_Cell, &AtmInfo dielec / BornZ
    // (unit_mod.f90:64-209; dielec defaults to 1.0 in every element) and &EwaldInfo
    // (EwaldParam.f90: decide_EwParam = .true., prec_Ew = 1e-6, Lmb = 0.8, Gmesh, Rmesh)
    bool force_dd = false, decide_ew = true;
    std::vector<int> sup_cell{5, 5, 5}, gmesh{0, 0, 0}, rmesh{0, 0, 0};
    std::vector<double> dielec(9, 1.0), born((size_t)9 * nb, 0.0);
    double prec_ew = 1e-6, lmb = 0.8;
    check(nml::get(fci, "Force_dd", force_dd));
    check(nml::get(cri, "Sup_Cell", {3}, sup_cell));
    check(nml::get(ati, "dielec", {3, 3}, dielec));
    check(nml::get(ati, "BornZ", {3, 3, nb}, born));
    double ew_lmb = 0.0;
    int ew_g[3] = {0, 0, 0}, ew_cnt[2] = {0, 0};
    if (force_dd) {
        if (!groups.count("ewaldinfo")) die("Force_dd = .true. needs the &EwaldInfo namelist (Rmesh)");
        const nml::Group& ewi = groups["ewaldinfo"];
        check(nml::get(ewi, "decide_EwParam", decide_ew));
        check(nml::get(ewi, "prec_Ew", prec_ew));
        check(nml::get(ewi, "Lmb", lmb));
        check(nml::get(ewi, "Gmesh", {3}, gmesh));
        check(nml::get(ewi, "Rmesh", {3}, rmesh));
        if (spring_ewald_setup(lat.data(), nb, pos.data(), dielec.data(), born.data(), decide_ew ? 1 : 0, prec_ew, lmb,
                               gmesh.data(), rmesh.data(), sup_cell.data(), &ew_lmb, ew_g, ew_cnt, nullptr, nullptr, 0))
            die(spring_host_last_error());
    }

    // ---- force constants
    const std::string tc = temp_char(T);
    // Point defects: &PointDefInfo (ReadPointDefVar, Helper_m.f90:135-307) with its defaults and checks
    const double FILL = 99999.0;
    const bool point_def = groups.count("pointdefinfo") > 0;
    std::string ifc2_pd = "FC2nd_" + prefix + tc + "K_F_pd.h5";
    std::vector<double> mass_def(mass);
    double rho_def = 1.0e-6;
    std::vector<int> qmesh_pd{7, 7, 7};
    bool mat_inv_full = true, optc_therm = true;
    if (point_def) {
        const nml::Group& pdi = groups["pointdefinfo"];
        std::vector<double> mdef_in(nb, FILL);
        std::vector<int> def_pos(nb, 0), cell_atom(4 * 5, (int)FILL);
        int numdef = 0;
        check(nml::get(pdi, "IFC2_file_pd", ifc2_pd));
        check(nml::get(pdi, "Mass_def", {nb}, mdef_in));
        check(nml::get(pdi, "rho_def", rho_def));
        check(nml::get(pdi, "qMesh_pd", {3}, qmesh_pd));
        check(nml::get(pdi, "def_pos", {nb}, def_pos));
        check(nml::get(pdi, "NumDef_sup", numdef));
        check(nml::get(pdi, "cell_atom", {4, 5}, cell_atom));
        check(nml::get(pdi, "MatInvFull", mat_inv_full));
        check(nml::get(pdi, "OptcTherm", optc_therm));
        if (std::all_of(def_pos.begin(), def_pos.end(), [](int v) { return v == 0; }))
            die("&PointDefInfo: def_pos (mandatory) is not provided");
        int cnt = 0;
        for (int mu = 0; mu < nb; ++mu)
            if (def_pos[mu] != 0) {
                if (std::fabs(mdef_in[cnt] - FILL) < 1e-8)
                    die("&PointDefInfo: def_pos names more defects than Mass_def gives masses");
                mass_def[mu] = mdef_in[cnt];
                mdef_in[cnt++] = 0.0;
            }
        for (int mu = 0; mu < nb; ++mu)
            if (!(mdef_in[mu] < 1e-8 || std::fabs(mdef_in[mu] - FILL) < 1e-8))
                die("&PointDefInfo: mismatch between def_pos and Mass_def");
        if (numdef <= 0) die("&PointDefInfo: NumDef_sup is 0");
        for (int k = 0; k < std::min(numdef, 5); ++k)
            for (int r = 0; r < 4; ++r)
                if (cell_atom[4 * k + r] == (int)FILL) die("&PointDefInfo: NumDef_sup and cell_atom do not match");
    }
    const Fc f2 = read_fc("FC2nd_" + prefix + tc + "K_F.h5", 2);
    const Fc f3 = read_fc("FC3rd_" + prefix + tc + "K_F.h5", 3);
    Fc f4;
    if (four) f4 = read_fc("FC4th_" + prefix + tc + "K_F.h5", 4);
    Fc f2pd;
    if (point_def) f2pd = read_fc(ifc2_pd, 2);
    for (const Fc* f : {&f2, &f3})
        if (f->nb != nb) die("FC file basis count differs from Nbasis");
    if (point_def && f2pd.nb != nb) die(ifc2_pd + ": basis count differs from Nbasis");
    const std::vector<int> rot = point_group(lat, pos, typ, nb, std::max(symprec, 1e-7));
    const int nrot = (int)rot.size() / 9;

    if (dry) {
        std::printf("{\"prefix\": \"%s\", \"T\": \"%s\", \"nbasis\": %d, \"mass\": [", prefix.c_str(), tc.c_str(), nb);
        for (int i = 0; i < nb; ++i) std::printf("%s%.10g", i ? ", " : "", mass[i]);
        std::printf("], \"latvec\": [");
        for (int i = 0; i < 9; ++i) std::printf("%s%.15g", i ? ", " : "", lat[i]);
        std::printf("], \"qmesh\": [%d, %d, %d], \"shift\": [%d, %d, %d], \"time_rev\": %d, \"sigma\": %.15g, ",
                    qmesh[0], qmesh[1], qmesh[2], shift[0], shift[1], shift[2], time_rev, sigma);
        std::printf("\"isotope\": %s, \"four_phonon\": %s, \"g2iso\": [", isotope ? "true" : "false", four ? "true" : "false");
        for (int i = 0; i < nb; ++i) std::printf("%s%.15g", i ? ", " : "", g2iso[i]);
        std::printf("], \"pol3\": [");
        for (size_t i = 0; i < pol3.size(); ++i) std::printf("%s%d", i ? ", " : "", pol3[i]);
        std::printf("], \"pol4\": [");
        for (size_t i = 0; i < pol4.size(); ++i) std::printf("%s%d", i ? ", " : "", pol4[i]);
        double s2 = 0, s3 = 0, s4 = 0;
        for (double v : f2.fc) s2 += v;
        for (double v : f3.fc) s3 += v * v;
        for (double v : f4.fc) s4 += v * v;
        std::printf("], \"na2\": %d, \"na3\": %d, \"na4\": %d, \"fc2_sum\": %.15g, \"fc3_sumsq\": %.15g, "
                    "\"fc4_sumsq\": %.15g, \"n_rotations\": %d, \"force_dd\": %s, \"ewald_lmb\": %.15g, "
                    "\"ewald_gmesh\": [%d, %d, %d], \"ewald_points\": [%d, %d], \"point_defect\": %s, "
                    "\"qmesh_pd\": [%d, %d, %d], \"rho_def\": %.15g, \"mat_inv_full\": %s, \"optc_therm\": %s, "
                    "\"ifc2_file_pd\": \"%s\", \"mass_def\": [",
                    f2.na, f3.na, four ? f4.na : 0, s2, s3, s4, nrot, force_dd ? "true" : "false", ew_lmb, ew_g[0],
                    ew_g[1], ew_g[2], ew_cnt[0], ew_cnt[1], point_def ? "true" : "false", qmesh_pd[0], qmesh_pd[1],
                    qmesh_pd[2], rho_def, mat_inv_full ? "true" : "false", optc_therm ? "true" : "false",
                    ifc2_pd.c_str());
        for (int i = 0; i < nb; ++i) std::printf("%s%.10g", i ? ", " : "", mass_def[i]);
        std::printf("]}\n");
        return 0;
    }

    // ---- the q0 loop of main.f90:552-715 in one call per term, then kappa
    spring_dims dims{};
    dims.nbasis = nb;
    for (int k = 0; k < 3; ++k) dims.mesh[k] = qmesh[k];
    dims.n_temps = 1;
    dims.device = -1;
    spring_ctx* c = nullptr;
    if (spring_ctx_create(&c, &dims)) die("cannot create a context (is a CUDA device present?)");
    gpu(c, spring_set_crystal(c, lat.data(), mass.data()));
    gpu(c, spring_set_fc2(c, f2.na, f2.num.data(), f2.idx.data(), f2.fc.data()));
    gpu(c, spring_set_fc3(c, f3.na, f3.num.data(), f3.idx.data(), f3.fc.data()));
    if (four) gpu(c, spring_set_fc4(c, f4.na, f4.num.data(), f4.idx.data(), f4.fc.data()));
    if (force_dd)
        gpu(c, spring_set_dipole(c, pos.data(), dielec.data(), born.data(), decide_ew ? 1 : 0, prec_ew, lmb,
                                 gmesh.data(), rmesh.data(), sup_cell.data()));
    gpu(c, spring_make_mesh(c, shift.data(), 1, nullptr, nullptr, nullptr));
    const int nq = qmesh[0] * qmesh[1] * qmesh[2];
    int nq0 = 0;
    std::vector<int> irr((size_t)3 * nq), posq(nq), mult(nq);
    gpu(c, spring_find_irr_q(c, nrot, rot.data(), time_rev, &nq0, irr.data(), posq.data(), mult.data()));
    gpu(c, spring_compute_phonons(c, &T, freq_cut));
    if (point_def)
        gpu(c, spring_set_point_defect(c, qmesh_pd.data(), f2pd.na, f2pd.num.data(), f2pd.idx.data(), f2pd.fc.data(),
                                       mass_def.data(), rho_def, mat_inv_full ? 1 : 0, optc_therm ? 1 : 0));
    std::vector<double> scat_pd(point_def ? (size_t)ndof * nq0 : 0, 0.0);
    const int prec = precision == "bf16x3" ? SPRING_BF16X3 : (precision == "bf16" ? SPRING_BF16 : SPRING_FP64);
    if (precision != "fp64" && precision != "bf16" && precision != "bf16x3") die("-precision: fp64, bf16 or bf16x3");
    gpu(c, spring_set_precision(c, prec));
    const int dm = delta == "gauss" ? SPRING_DELTA_GAUSS : SPRING_DELTA_TETRA;
    std::vector<double> lw_all((size_t)ndof * nq0, 0.0), omega((size_t)ndof * nq0), p3((size_t)ndof * nq0, 0.0);
    gpu(c, spring_reset_linewidths(c));
    // Restart (main.f90:502-545, 630-713): LW_Allq0 of the points already done comes from the
    // restart file, and the loop starts after them; with WriteRestart the file is rewritten after
    // every block of points.
    const std::string rdir = "Restart_" + prefix, rfile = rdir + "/" + prefix + tc + "K_LW_Restart.h5";
    int start = 1;
    if (rrestart) {
        int prog[2] = {0, 0};
        if (spring_h5_read_restart(rfile.c_str(), ndof, nq0, prog, lw_all.data())) die(spring_host_last_error());
        start = prog[1] == 1 ? prog[0] + 1 : std::max(1, prog[0]);
        for (int q = start - 1; q < nq0; ++q)
            for (int s = 0; s < ndof; ++s) lw_all[(size_t)ndof * q + s] = 0.0;  // recomputed below
        gpu(c, spring_set_linewidths(c, lw_all.data()));
        std::printf("restart: %d of %d irreducible points read from %s\n", start - 1, nq0, rfile.c_str());
    }
    if (wrestart) mkdir(rdir.c_str(), 0755);
    const int block = wrestart ? std::max(1, (nq0 + 15) / 16) : nq0;
    for (int i0 = start; i0 <= nq0; i0 += block) {
        const int n = std::min(block, nq0 - i0 + 1);
        std::vector<double> p3b((size_t)ndof * n);
        gpu(c, spring_linewidth3(c, i0, n, dm, sigma, pol3.data(), nullptr, p3b.data()));
        std::copy(p3b.begin(), p3b.end(), p3.begin() + (size_t)ndof * (i0 - 1));
        if (isotope) gpu(c, spring_linewidth_iso(c, i0, n, dm, sigma, g2iso.data(), nullptr));
        if (four) gpu(c, spring_linewidth4(c, i0, n, dm, sigma, pol4.data(), nullptr));
        if (point_def) gpu(c, spring_linewidth_pd(c, i0, n, scat_pd.data() + (size_t)ndof * (i0 - 1), 1));
        if (wrestart) {
            gpu(c, spring_get_linewidths(c, lw_all.data()));
            if (spring_h5_write_restart(rfile.c_str(), ndof, nq0, i0 + n - 1, 1, lw_all.data()))
                die(spring_host_last_error());
        }
    }
    gpu(c, spring_get_linewidths(c, lw_all.data()));
    gpu(c, spring_get_phonons(c, 1, nullptr, omega.data(), nullptr, nullptr, nullptr));
    // branch window of the kappa sum: Polarization3rd (and 4th) first rows
    int srange[2] = {pol3[0], pol3[1]};
    for (int k = 1; k < 3; ++k) {
        srange[0] = std::min(srange[0], pol3[2 * k]);
        srange[1] = std::max(srange[1], pol3[2 * k + 1]);
    }
    std::vector<double> kappa(9), modek((size_t)9 * ndof);
    std::vector<double> rxyz;
    if (symm) {  // Rxyz = L W L^-1 (Symmetry_m.f90:92-97), Fortran Rxyz(3,3,nsym)
        double Lm[3][3], Li[3][3];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) Lm[r][k] = lat[r + 3 * k];
        const double det = Lm[0][0] * (Lm[1][1] * Lm[2][2] - Lm[1][2] * Lm[2][1]) -
                           Lm[0][1] * (Lm[1][0] * Lm[2][2] - Lm[1][2] * Lm[2][0]) +
                           Lm[0][2] * (Lm[1][0] * Lm[2][1] - Lm[1][1] * Lm[2][0]);
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k) {
                const int r1 = (k + 1) % 3, r2 = (k + 2) % 3, c1 = (r + 1) % 3, c2 = (r + 2) % 3;
                Li[r][k] = (Lm[r1][c1] * Lm[r2][c2] - Lm[r1][c2] * Lm[r2][c1]) / det;
            }
        rxyz.resize((size_t)9 * nrot);
        for (int s = 0; s < nrot; ++s) {
            const int* W = &rot[9 * s];
            for (int r = 0; r < 3; ++r)
                for (int k = 0; k < 3; ++k) {
                    double v = 0.0;
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) v += Lm[r][a] * W[3 * a + b] * Li[b][k];
                    rxyz[(size_t)9 * s + r + 3 * k] = v;
                }
        }
    }
    gpu(c, spring_kappa_rta(c, symm ? 1 : 0, symm ? nrot : 0, symm ? rxyz.data() : nullptr, srange, kappa.data(),
                            mode_k ? modek.data() : nullptr));
    spring_ctx_destroy(c);

    // ---- outputs
    const std::string kfile = "kappa_" + prefix + tc + "K.h5", afile = "linewidth_IBZ_" + prefix + tc + "K.txt";
    std::vector<double> lwo((size_t)2 * ndof * nq0), p3o((size_t)2 * ndof * nq0);
    for (int q = 0; q < nq0; ++q)
        for (int s = 0; s < ndof; ++s) {
            lwo[(size_t)2 * ndof * q + s] = p3o[(size_t)2 * ndof * q + s] = omega[(size_t)ndof * q + s];
            lwo[(size_t)2 * ndof * q + ndof + s] = lw_all[(size_t)ndof * q + s];
            // P_Allq0 = P_q0 * 1000 / (9 Ndof^2 Nq1points), in fs (main.f90:687)
            p3o[(size_t)2 * ndof * q + ndof + s] = p3[(size_t)ndof * q + s] * 1000.0 / (9.0 * ndof * ndof * (double)nq);
        }
    std::vector<double> pdo;
    if (point_def) {  // Scatter_pd: omega alongside the rates (w2dh5_no_grp_type2, main.f90:778)
        pdo.resize((size_t)2 * ndof * nq0);
        for (int q = 0; q < nq0; ++q)
            for (int s = 0; s < ndof; ++s) {
                pdo[(size_t)2 * ndof * q + s] = omega[(size_t)ndof * q + s];
                pdo[(size_t)2 * ndof * q + ndof + s] = scat_pd[(size_t)ndof * q + s];
            }
    }
    if (spring_h5_write_kappa(kfile.c_str(), kappa.data(), ndof, nq0, lwo.data(), p3o.data(),
                              mode_k ? modek.data() : nullptr, point_def ? pdo.data() : nullptr))
        die(spring_host_last_error());
    if (point_def) {  // ScatterRate_pd_IBZ_<prefix><T>K.txt (WriteAsciiOutFile, main.f90:669-670)
        const std::string pfile = "ScatterRate_pd_IBZ_" + prefix + tc + "K.txt";
        FILE* fp = std::fopen(pfile.c_str(), "w");
        if (!fp) die("cannot write " + pfile);
        std::fprintf(fp, "#--------- phonon_frequency(rad.THz) ( %4d columns) ---------      ---------- scattering "
                         "rate(1/ps) ( %4d columns) ----------\n", ndof, ndof);
        for (int q = 0; q < nq0; ++q) {
            std::string line;
            for (int s = 0; s < ndof; ++s) line += g20(omega[(size_t)ndof * q + s]) + "  ";
            for (int s = 0; s < ndof; ++s) line += g20(scat_pd[(size_t)ndof * q + s]) + (s + 1 < ndof ? "  " : "");
            std::fprintf(fp, "%s\n", line.c_str());
        }
        std::fclose(fp);
    }
    FILE* fa = std::fopen(afile.c_str(), "w");
    if (!fa) die("cannot write " + afile);
    std::fprintf(fa, "#--------- phonon_frequency(rad.THz) ( %4d columns) ---------      ---------- linewidth(rad.THz) "
                     "( %4d columns) ----------\n", ndof, ndof);
    for (int q = 0; q < nq0; ++q) {
        std::string line;
        for (int s = 0; s < ndof; ++s) line += g20(omega[(size_t)ndof * q + s]) + "  ";
        for (int s = 0; s < ndof; ++s) line += g20(lw_all[(size_t)ndof * q + s]) + (s + 1 < ndof ? "  " : "");
        std::fprintf(fa, "%s\n", line.c_str());
    }
    std::fclose(fa);
    std::printf("kappa (W/m/K): %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e %.6e\n", kappa[0], kappa[1], kappa[2], kappa[3],
                kappa[4], kappa[5], kappa[6], kappa[7], kappa[8]);
    std::printf("Thermal conductivity information written in file: %s\n", kfile.c_str());
    return 0;
}
