// The solver's printed outputs, in the reference's file names and layouts
// (host code; the functions read the context's results of the last solve):
//
//  * print_impG / print_impSigma / print_impG0 (ED_IO/print_impG.f90:38-46,
//    print_impSigma.f90:37-45, print_impG0.f90:37-45), normal bath: per spin
//    s and orbital a the files <name>_l<a><a>_s<s>_iw<suffix>.ed (Lmats
//    points) and <name>_l<a><a>_s<s>_realw<suffix>.ed (Lreal points), <name>
//    impG, impSigma, and impG again for G0 (print_impG0_normal writes the
//    Weiss field under the impG names, so it replaces print_impG's files).
//    The files are written by SciFortran's splot (SF_IOTOOLS, not in the
//    tree, no version pinned): one line per point, the abscissa, Im f, Re f.
//    The numbers here are ES24.16 (17 significant digits: read back, they
//    give the same doubles); the reference reads these files list-directed
//    (sread), so any numeric layout of the three columns reads the same.
//  * read_impSigma (ED_IO/read_impSigma.f90:38-46): the self-energy files
//    read back into the context.
//  * write_legend / write_observables (ED_OBSERVABLES.f90:715-849, called by
//    observables_impurity at :418-420) and write_energy_info / write_energy
//    (:760-774, :851-857, called by local_energy_impurity at :681-684), with
//    their Fortran edit descriptors.
//
// ed_file_suffix (ED_MAIN.f90:185,193,214): "" for one impurity, the site
// suffix in the lattice solvers; passed by the caller.  dir: the directory
// the files go to ("" or null: the working directory, as the reference).
#include <cmath>
#include <complex>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fortfmt.h"
#include "internal.cuh"

using namespace dmfted;

namespace {

int ok() { return set_error(DMFTED_OK, ""); }

std::string in_dir(const char *dir, const std::string &name) {
    if (!dir || !*dir) return name;
    std::string d(dir);
    if (d.back() != '/') d += '/';
    return d + name;
}

std::string suffix_of(const char *s) { return s ? std::string(s) : std::string(); }

void write_file(const std::string &path, const std::string &text, bool append) {
    std::FILE *f = std::fopen(path.c_str(), append ? "a" : "w");
    DM_REQUIRE(f, DMFTED_ERR_ARG, "cannot open " + path);
    const size_t w = std::fwrite(text.data(), 1, text.size(), f);
    const int cl = std::fclose(f);
    DM_REQUIRE(w == text.size() && cl == 0, DMFTED_ERR_ARG, "write failed on " + path);
}

// The (spin, orbital) block so = ispin*norb + iorb of a device array of
// complex (nspin, norb, L) blocks.
std::vector<std::complex<double>> block(const DBuf<double> &d, int so, int L) {
    std::vector<std::complex<double>> h((size_t)std::max(L, 0));
    if (L > 0)
        DM_CUDA(cudaMemcpy(h.data(), d.p + 2 * (size_t)so * L, (size_t)L * 2 * sizeof(double),
                           cudaMemcpyDeviceToHost));
    return h;
}

// wm = pi/beta (2n-1), wr = linspace(wini, wfin, Lreal) (print_impG.f90:7-9)
std::vector<double> matsubara(const dmfted_params &p) {
    std::vector<double> w((size_t)std::max(p.lmats, 0));
    for (int i = 0; i < p.lmats; i++) w[i] = M_PI / p.beta * (2.0 * (i + 1) - 1.0);
    return w;
}
std::vector<double> real_axis(const dmfted_params &p) {
    std::vector<double> w((size_t)std::max(p.lreal, 0));
    for (int i = 0; i < p.lreal; i++)
        w[i] = p.lreal > 1 ? p.wini + (p.wfin - p.wini) * i / (double)(p.lreal - 1) : p.wini;
    return w;
}

std::string splot_text(const std::vector<double> &x, const std::vector<std::complex<double>> &y) {
    std::string out;
    out.reserve(x.size() * 76);
    for (size_t i = 0; i < x.size(); i++) {
        fort::Record r;
        r.add(fort::ES(x[i], 24, 16)).add(fort::ES(y[i].imag(), 24, 16)).add(fort::ES(y[i].real(), 24, 16));
        out += r.s + "\n";
    }
    return out;
}

std::string gf_name(const std::string &name, int iorb, int ispin, const char *axis,
                    const std::string &sfx) {
    return name + "_l" + std::to_string(iorb + 1) + std::to_string(iorb + 1) + "_s" +
           std::to_string(ispin + 1) + "_" + axis + sfx + ".ed";
}

void print_pair(dmfted_ctx *c, const char *dir, const char *suffix, const std::string &name,
                const DBuf<double> &mats, const DBuf<double> &real) {
    DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
    const dmfted_params &p = c->p;
    const std::vector<double> wm = matsubara(p), wr = real_axis(p);
    const std::string sfx = suffix_of(suffix);
    for (int is = 0; is < c->nspin; is++)
        for (int a = 0; a < c->norb; a++) {
            const int so = is * c->norb + a;
            write_file(in_dir(dir, gf_name(name, a, is, "iw", sfx)),
                       splot_text(wm, block(mats, so, p.lmats)), false);
            write_file(in_dir(dir, gf_name(name, a, is, "realw", sfx)),
                       splot_text(wr, block(real, so, p.lreal)), false);
        }
}

// sread of one file of L points: x, Im f, Re f per line, list-directed.
std::vector<std::complex<double>> sread(const std::string &path, int L) {
    std::ifstream in(path);
    DM_REQUIRE(in.good(), DMFTED_ERR_ARG, "read_impSigma: cannot open " + path);
    std::vector<std::complex<double>> y((size_t)std::max(L, 0));
    for (int i = 0; i < L; i++) {
        double x, im, re;
        in >> x >> im >> re;
        DM_REQUIRE(!in.fail(), DMFTED_ERR_ARG,
                   "read_impSigma: " + path + " ends before point " + std::to_string(i + 1) +
                       " of " + std::to_string(L));
        y[i] = {re, im};
    }
    return y;
}

// Label of write_legend: the column number followed by the name.
std::string lab(int col, const std::string &name) { return std::to_string(col) + name; }

}  // namespace

extern "C" {

int dmfted_print_impg(dmfted_ctx *c, const char *dir, const char *suffix) {
    try {
        DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
        print_pair(c, dir, suffix, "impG", c->gm, c->gr);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_print_impsigma(dmfted_ctx *c, const char *dir, const char *suffix) {
    try {
        DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
        print_pair(c, dir, suffix, "impSigma", c->sm, c->sr);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_print_impg0(dmfted_ctx *c, const char *dir, const char *suffix) {
    try {
        DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
        print_pair(c, dir, suffix, "impG", c->g0m, c->g0r);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_read_impsigma(dmfted_ctx *c, const char *dir, const char *suffix) {
    try {
        DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
        DM_CUDA(cudaSetDevice(c->device));
        const dmfted_params &p = c->p;
        const std::string sfx = suffix_of(suffix);
        const size_t gsz = (size_t)c->nspin * c->norb;
        // every file is read before the context's arrays change
        std::vector<std::vector<std::complex<double>>> m(gsz), r(gsz);
        for (int is = 0; is < c->nspin; is++)
            for (int a = 0; a < c->norb; a++) {
                const int so = is * c->norb + a;
                m[so] = sread(in_dir(dir, gf_name("impSigma", a, is, "iw", sfx)), p.lmats);
                r[so] = sread(in_dir(dir, gf_name("impSigma", a, is, "realw", sfx)), p.lreal);
            }
        c->sm.alloc(std::max<size_t>(2 * gsz * p.lmats, 2));
        c->sr.alloc(std::max<size_t>(2 * gsz * p.lreal, 2));
        c->sigma_now.assign(2 * gsz, 0.0);
        for (size_t so = 0; so < gsz; so++) {
            if (p.lmats > 0)
                DM_CUDA(cudaMemcpy(c->sm.p + 2 * so * p.lmats, m[so].data(),
                                   (size_t)p.lmats * 2 * sizeof(double), cudaMemcpyHostToDevice));
            if (p.lreal > 0)
                DM_CUDA(cudaMemcpy(c->sr.p + 2 * so * p.lreal, r[so].data(),
                                   (size_t)p.lreal * 2 * sizeof(double), cudaMemcpyHostToDevice));
            if (p.lmats >= 2) {
                c->sigma_now[2 * so] = m[so][0].imag();
                c->sigma_now[2 * so + 1] = m[so][1].imag();
            }
        }
        c->sigma_read = true;
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_write_observables(dmfted_ctx *c, const char *dir, const char *suffix, int32_t legend) {
    try {
        DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
        DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
        const dmfted_params &p = c->p;
        const int no = c->norb, ns = c->nspin;
        const std::string sfx = suffix_of(suffix);
        if (legend) {
            // write_legend, normal mode (:720-731): "(A1,90(A10,6X))"
            fort::Record h("      ");
            auto put = [&](const std::string &l) { h.add(fort::A(l, 10)); };
            for (int a = 1; a <= no; a++) put(lab(a, "dens_" + std::to_string(a)));
            for (int a = 1; a <= no; a++) put(lab(no + a, "docc_" + std::to_string(a)));
            for (int a = 1; a <= no; a++) put(lab(2 * no + a, "nup_" + std::to_string(a)));
            for (int a = 1; a <= no; a++) put(lab(3 * no + a, "ndw_" + std::to_string(a)));
            for (int a = 1; a <= no; a++) put(lab(4 * no + a, "mag_" + std::to_string(a)));
            put(lab(5 * no + 1, "s2"));
            put(lab(5 * no + 2, "egs"));
            for (int a = 1; a <= no; a++)
                for (int b = 1; b <= no; b++)
                    put(lab(5 * no + 2 + (a - 1) * no + b,
                            "sz2_" + std::to_string(a) + std::to_string(b)));
            for (int a = 1; a <= no; a++)
                for (int b = 1; b <= no; b++)
                    put(lab((5 + no) * no + 2 + (a - 1) * no + b,
                            "n2_" + std::to_string(a) + std::to_string(b)));
            // the z and sig column numbers step by Nspin per spin, as written
            for (int s = 1; s <= ns; s++)
                for (int a = 1; a <= no; a++)
                    put(lab((5 + 2 * no) * no + 2 + (s - 1) * ns + a,
                            "z_" + std::to_string(a) + "s" + std::to_string(s)));
            for (int s = 1; s <= ns; s++)
                for (int a = 1; a <= no; a++)
                    put(lab((6 + 2 * no) * no + 2 + ns + (s - 1) * ns + a,
                            "sig_" + std::to_string(a) + "s" + std::to_string(s)));
            write_file(in_dir(dir, "observables_info.ed"), "#" + h.s + "\n", false);
            // parameters_info.ed (:751-756): "(A1,90(A14,1X))"
            fort::Record q;
            q.add(fort::A("1xmu", 14)).add(fort::A("2beta", 14));
            for (int a = 1; a <= no; a++) q.add(fort::A(lab(2 + a, "U_" + std::to_string(a)), 14));
            q.add(fort::A(lab(2 + no + 1, "U'"), 14)).add(fort::A(lab(2 + no + 2, "Jh"), 14));
            write_file(in_dir(dir, "parameters_info.ed"), "#" + q.s + "\n", false);
        }
        // get_szr (:695-708) on the self-energy the solve's observables saw
        std::vector<double> zimp((size_t)no * ns), simp((size_t)no * ns);
        const double wm1 = M_PI / p.beta, wm2 = 3.0 * M_PI / p.beta;
        for (int s = 0; s < ns; s++)
            for (int a = 0; a < no; a++) {
                const size_t so = (size_t)s * no + a;
                const double s1 = c->szr_sigma.size() > 2 * so ? c->szr_sigma[2 * so] : 0.0;
                const double s2 = c->szr_sigma.size() > 2 * so + 1 ? c->szr_sigma[2 * so + 1] : 0.0;
                simp[so] = s1 - wm1 * (s2 - s1) / (wm2 - wm1);
                zimp[so] = 1.0 / (1.0 + std::fabs(s1 / wm1));
            }
        // write_observables, normal mode (:786-797): "(90(F15.9,1X))"
        fort::Record v;
        auto val = [&](double x) { v.add(fort::F(x, 15, 9)); };
        for (int k = 0; k < 5; k++) {
            // dens, docc, dens_up, dens_dw, magz; c->obs holds dens, up, dw, docc, magz
            static const int order[5] = {0, 3, 1, 2, 4};
            for (int a = 0; a < no; a++) val(c->obs[order[k] * no + a]);
        }
        val(c->s2tot);
        val(c->egs);
        for (int a = 0; a < no; a++)
            for (int b = 0; b < no; b++) val(c->sz2[a * no + b]);
        for (int a = 0; a < no; a++)
            for (int b = 0; b < no; b++) val(c->n2[a * no + b]);
        for (int s = 0; s < ns; s++)
            for (int a = 0; a < no; a++) val(zimp[(size_t)s * no + a]);
        for (int s = 0; s < ns; s++)
            for (int a = 0; a < no; a++) val(simp[(size_t)s * no + a]);
        write_file(in_dir(dir, "observables_all" + sfx + ".ed"), v.s + "\n", true);
        write_file(in_dir(dir, "observables_last" + sfx + ".ed"), v.s + "\n", false);
        // parameters_last (:815-817): "(90F15.9)", no separator
        fort::Record pl("");
        pl.add(fort::F(p.xmu, 15, 9)).add(fort::F(p.beta, 15, 9));
        for (int a = 0; a < no; a++) pl.add(fort::F(p.uloc[a], 15, 9));
        pl.add(fort::F(p.ust, 15, 9)).add(fort::F(p.jh, 15, 9)).add(fort::F(p.jx, 15, 9));
        pl.add(fort::F(p.jp, 15, 9));
        write_file(in_dir(dir, "parameters_last" + sfx + ".ed"), pl.s + "\n", false);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_write_energy(dmfted_ctx *c, const char *dir, const char *suffix) {
    try {
        DM_REQUIRE(c, DMFTED_ERR_ARG, "null context");
        DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
        // write_energy_info (:760-774): "(A1,90(A14,1X))"
        static const char *names[8] = {"<Hi>",  "<V>=<Hi-Ehf>", "<Eloc>", "<Ehf>",
                                       "<Dst>", "<Dnd>",        "<Dse>",  "<Dph>"};
        fort::Record h;
        for (int k = 0; k < 8; k++) h.add(fort::A(lab(k + 1, names[k]), 14));
        write_file(in_dir(dir, "energy_info.ed"), "#" + h.s + "\n", false);
        // write_energy (:851-857): "(90F15.9)" Epot, Epot-Ehartree, Eknot,
        // Ehartree, Dust, Dund, Dse, Dph; c->eloc = {Epot, Eint, Ehartree,
        // Eknot, Dust, Dund, Dse, Dph}
        const std::vector<double> &e = c->eloc;
        fort::Record r("");
        for (double x : {e[0], e[0] - e[2], e[3], e[2], e[4], e[5], e[6], e[7]})
            r.add(fort::F(x, 15, 9));
        write_file(in_dir(dir, "energy_last" + suffix_of(suffix) + ".ed"), r.s + "\n", false);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

}  // extern "C"
