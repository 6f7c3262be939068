// The solver's files that let a DMFT run resume across the Fortran / device
// boundary, in the reference's text formats:
//
//  * the bath file hamiltonian.restart / hamiltonian.used: write_dmft_bath
//    (ED_BATH/dmft_aux.f90:310-336, normal bath): one header line of
//    "(90(A21,1X))" labels #Ek_l<a>_s<s>, Vk_l<a>_s<s>, then Nbath rows of
//    "(90(F21.12,1X))" values ((e(s,a,k), v(s,a,k), a=1..Norb), s=1..Nspin);
//    read back by init_dmft_bath (:158-180): the header skipped, then
//    min(lines, Nbath) rows read list-directed;
//  * the state list state_list.ed: print_state_list (ED_DIAG.f90:258-264,
//    401-445), one header line, then per state
//    "(i3,f18.12,2x,ES19.12,1x,2i3,3x,i3,i10)": i, E_i,
//    exp(-beta (E_i - E_min)), nup, ndw, sector, dimension;  read back as
//    state_list.restart by setup_pointers_normal (ED_SETUP.f90:403-425):
//    lanc_nstates_total = the file's line count, neigen_sector(s) =
//    max(1, number of listed states of sector s), every listed nup/ndw checked
//    against its sector.
//
// Host code only: the bath files need no device, the state list is the
// eigenspace of the context's last solve.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fortfmt.h"
#include "internal.cuh"

using namespace dmfted;

namespace {

int ok() { return set_error(DMFTED_OK, ""); }

using fort::A;
using fort::ES;
using fort::F;
using fort::I;

void check_bath_dims(const dmfted_params *p, int32_t nb) {
    DM_REQUIRE(p->norb >= 1 && p->nspin >= 1 && p->nbath >= 0, DMFTED_ERR_ARG, "bad dimensions");
    DM_REQUIRE(nb == 2 * p->nspin * p->norb * p->nbath, DMFTED_ERR_ARG,
               "set_dmft_bath error: wrong bath dimensions");
}

// e(s,a,k) / v(s,a,k) of the set_dmft_bath array layout
// (ED_BATH/dmft_aux.f90:493-512): io = k + a*Nbath + s*Nbath*Norb.
inline int64_t bath_io(const dmfted_params *p, int s, int a, int k) {
    return k + (int64_t)a * p->nbath + (int64_t)s * p->nbath * p->norb;
}

}  // namespace

extern "C" {

int dmfted_save_bath(const dmfted_params *p, const char *path, const double *bath, int32_t nb) {
    try {
        DM_REQUIRE(p && path && bath, DMFTED_ERR_ARG, "null argument");
        check_bath_dims(p, nb);
        const int64_t half = (int64_t)nb / 2;
        fort::Record head;
        for (int s = 0; s < p->nspin; s++)
            for (int a = 0; a < p->norb; a++) {
                const std::string tag = "l" + std::to_string(a + 1) + "_s" + std::to_string(s + 1);
                head.add(A("#Ek_" + tag, 21)).add(A("Vk_" + tag, 21));
            }
        std::string out = head.s + "\n";
        for (int k = 0; k < p->nbath; k++) {
            fort::Record row;
            for (int s = 0; s < p->nspin; s++)
                for (int a = 0; a < p->norb; a++) {
                    const int64_t io = bath_io(p, s, a, k);
                    row.add(F(bath[io], 21, 12)).add(F(bath[half + io], 21, 12));
                }
            out += row.s + "\n";
        }
        std::FILE *f = std::fopen(path, "w");
        DM_REQUIRE(f, DMFTED_ERR_ARG, std::string("save_dmft_bath: cannot open ") + path);
        const size_t w = std::fwrite(out.data(), 1, out.size(), f);
        const int cl = std::fclose(f);
        DM_REQUIRE(w == out.size() && cl == 0, DMFTED_ERR_ARG,
                   std::string("save_dmft_bath: write failed on ") + path);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_read_bath(const dmfted_params *p, const char *path, double *bath, int32_t nb) {
    try {
        DM_REQUIRE(p && path && bath, DMFTED_ERR_ARG, "null argument");
        check_bath_dims(p, nb);
        std::ifstream in(path);
        DM_REQUIRE(in.good(), DMFTED_ERR_ARG, std::string("read bath: cannot open ") + path);
        std::vector<std::string> lines;
        for (std::string l; std::getline(in, l);) lines.push_back(l);
        const int64_t half = (int64_t)nb / 2;
        const int nrow = std::min<int>((int)lines.size(), p->nbath);
        for (int k = 0; k < nrow; k++) {
            DM_REQUIRE(k + 1 < (int)lines.size(), DMFTED_ERR_ARG,
                       std::string("read bath: end of file in ") + path);
            std::istringstream row(lines[k + 1]);
            for (int s = 0; s < p->nspin; s++)
                for (int a = 0; a < p->norb; a++) {
                    double e, v;
                    row >> e >> v;
                    DM_REQUIRE(!row.fail(), DMFTED_ERR_ARG,
                               std::string("read bath: bad row ") + std::to_string(k + 2) +
                                   " in " + path);
                    const int64_t io = bath_io(p, s, a, k);
                    bath[io] = e;
                    bath[half + io] = v;
                }
        }
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_print_state_list(dmfted_ctx *c, const char *path) {
    try {
        DM_REQUIRE(c && path, DMFTED_ERR_ARG, "null argument");
        DM_REQUIRE(c->solved, DMFTED_ERR_STATE, "no solve has run on this context");
        double emin = c->states.empty() ? 0.0 : c->states.front().e;
        for (const auto &st : c->states) emin = std::min(emin, st.e);
        std::string out = "# i       E_i           exp(-(E-E0)/T)       nup ndw  Sect     Dim\n";
        for (size_t i = 0; i < c->states.size(); i++) {
            const auto &st = c->states[i];
            const int is = st.isector;
            out += I((long long)i + 1, 3) + F(st.e, 18, 12) + "  " +
                   ES(std::exp(-c->p.beta * (st.e - emin)), 19, 12) + " " +
                   I(c->getnup[is - 1], 3) + I(c->getndw[is - 1], 3) + "   " + I(is, 3) +
                   I(c->getdim[is - 1], 10) + "\n";
        }
        std::FILE *f = std::fopen(path, "w");
        DM_REQUIRE(f, DMFTED_ERR_ARG, std::string("print_state_list: cannot open ") + path);
        const size_t w = std::fwrite(out.data(), 1, out.size(), f);
        const int cl = std::fclose(f);
        DM_REQUIRE(w == out.size() && cl == 0, DMFTED_ERR_ARG,
                   std::string("print_state_list: write failed on ") + path);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

int dmfted_read_state_list(dmfted_ctx *c, const char *path) {
    try {
        DM_REQUIRE(c && path, DMFTED_ERR_ARG, "null argument");
        std::ifstream in(path);
        DM_REQUIRE(in.good(), DMFTED_ERR_ARG, std::string("state list: cannot open ") + path);
        std::vector<std::string> lines;
        for (std::string l; std::getline(in, l);) lines.push_back(l);
        const int list_len = (int)lines.size();
        std::vector<int> count(c->nsectors, 0);
        for (int i = 1; i < list_len; i++) {
            std::istringstream row(lines[i]);
            long long istate, nup, ndw, isector, dim;
            double e, w;
            row >> istate >> e >> w >> nup >> ndw >> isector >> dim;
            if (row.fail()) break;  // the reference's read loop stops at the first failed read
            DM_REQUIRE(isector >= 1 && isector <= c->nsectors, DMFTED_ERR_ARG,
                       "setup_pointers_normal error: sector out of range in " + std::string(path));
            DM_REQUIRE(nup == c->getnup[isector - 1] && ndw == c->getndw[isector - 1], DMFTED_ERR_ARG,
                       "setup_pointers_normal error: nup!=getnup(isector).OR.ndw!=getndw(isector) ");
            count[isector - 1]++;
        }
        c->nstates_total = std::max(list_len, 1);
        for (int s = 0; s < c->nsectors; s++) c->neigen_sector[s] = std::max(1, count[s]);
    } catch (const StatusError &e) {
        return set_error(e.code, e.msg);
    }
    return ok();
}

}  // extern "C"
