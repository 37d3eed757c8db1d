// The main program of the reference's 3-D drivers over the C ABI: a deck in,
// the reference's output files out.
//
// Mirrors PROGRAM ratestate (fortran/3d/src/ratestate.f90:170-372) and PROGRAM
// viscouscycles (fortran/3d/src/viscouscycles.f90): buildG, buildO, the
// initial state, dt = 1e-3, then iterations of {export, exportPoints, RKQSm}
// until the time interval is reached or maximumIterations have run.  The
// iterations run on the device (ucg_run) in chunks; the recorder keeps one
// record per iteration in a device ring that is drained between chunks and
// written here, line for line in the reference's formats:
//   time.txt               "#  time  dt" header, (0, dt) at start, then per
//                          iteration (time, dt_done)          ES19.12E2 x 2
//   patch-%08d.dat         per iteration time, state, rate of one patch
//   volume-%08d.dat        (viscouscycles) of one volume    ES19.12E2, ES20.12E3 x 2 dgf
//   opts-<name>.dat        per iteration time and displacement (total; with
//                          volumes also faulting and flow)   ES19.12E2 x 4 or 10
// and, with verbose, the progress line every 50 iterations and the final
// iteration count on standard output.  Geometry files for visualisation
// (exportGeometry) are not written.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/ucg.h"

namespace {

// Fortran ESw.dEe edit descriptor (finite values, NaN and infinities as
// gfortran writes them), right-justified in w columns.
void put_es(std::string &out, double v, int w, int d, int e)
{
    std::string s;
    if (std::isnan(v)) {
        s = "NaN";
    } else if (std::isinf(v)) {
        s = v < 0 ? "-Infinity" : "Infinity";
        if ((int)s.size() > w) s = v < 0 ? "-Inf" : "Inf";
    } else {
        char buf[64];
        std::snprintf(buf, sizeof buf, "%.*E", d, v);
        char *ep = std::strchr(buf, 'E');
        const int x = std::atoi(ep + 1);
        *ep = '\0';
        const int ax = std::abs(x);
        int lim = 1;
        for (int k = 0; k < e; k++) lim *= 10;
        char xb[16];
        // an exponent wider than e digits fills the field with asterisks
        if (ax >= lim) {
            out.append(w, '*');
            return;
        }
        std::snprintf(xb, sizeof xb, "E%c%0*d", x < 0 ? '-' : '+', e, ax);
        s = std::string(buf) + xb;
    }
    if ((int)s.size() > w) s = std::string(w, '*');
    out.append(w - s.size(), ' ');
    out += s;
}

struct Out {
    FILE *f = nullptr;
    ~Out()
    {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" int ucg_deck_run(const ucg_deck *deck, const ucg_run_options *opt, long *iterations, double *time_out)
{
    if (!deck || !opt) return UCG_E_BADARG;
    if (opt->chunk < 1 || opt->maximum_iterations < 0 || !(opt->epsilon > 0.0)) return UCG_E_BADARG;
    ucg_deck_info info;
    ucg_deck_summary(deck, &info);
    const std::string wdir = opt->wdir ? opt->wdir : ucg_deck_wdir(deck);
    ucg_ctx *c = nullptr;
    int rc = ucg_deck_create(deck, opt->device, &c);
    if (rc) return rc;
    struct Guard {
        ucg_ctx *c;
        ~Guard() { ucg_destroy(c); }
    } guard{c};
    if ((rc = ucg_set_tolerance(c, opt->epsilon, opt->maximum_step))) return rc;
    if (opt->precision == UCG_PREC_HMATRIX || opt->precision == UCG_PREC_HMATRIX_SPLIT) {
        // hierarchical K only: the dense K is never assembled
        const double eta = opt->hm_eta > 0.0 ? opt->hm_eta : 2.0;
        const double eps = opt->hm_eps > 0.0 ? opt->hm_eps : 1.0e-6;
        const int leaf = opt->hm_leaf > 0 ? opt->hm_leaf : 32;
        if ((rc = ucg_build_hmatrix(c, opt->okada_mode, eta, eps, leaf))) return rc;
    } else if ((rc = ucg_assemble(c, opt->okada_mode))) {
        return rc;
    }
    if (opt->precision != UCG_PREC_FP64 && (rc = ucg_set_precision(c, opt->precision))) return rc;
    const int nobs = info.n_obs_point;
    if (nobs > 0 && (rc = ucg_build_O(c, opt->okada_mode))) return rc;
    const long len = ucg_state_len(c);
    std::vector<double> y(len);
    if ((rc = ucg_deck_init_state(deck, c, y.data()))) return rc;
    double dt_next = 1.0e-3;
    if ((rc = ucg_set_state(c, y.data(), 0.0, dt_next))) return rc;

    // observation states: element indices (1-based) -> 0-based for the recorder
    const int nst = info.n_obs_state;
    std::vector<int> st1(nst), st0(nst);
    ucg_deck_get_int(deck, "obs.state", st1.data(), nst);
    const int np = info.n_rect + info.n_tri;
    for (int j = 0; j < nst; j++) st0[j] = st1[j] - 1;
    const long cap = opt->chunk + 1;
    if ((rc = ucg_record(c, 1, st0.data(), nst, cap))) return rc;
    const long rlen = ucg_record_len(c);
    int per_point = 3;
    ucg_observation_info(c, nullptr, &per_point, nullptr);

    // output files
    Out ftime;
    std::vector<Out> fst(nst), fpt(nobs);
    auto open = [&](Out &o, const std::string &name) -> bool {
        o.f = std::fopen((wdir + "/" + name).c_str(), "w");
        return o.f != nullptr;
    };
    if (!open(ftime, "time.txt")) return UCG_E_BADARG;
    for (int j = 0; j < nst; j++) {
        char name[64];
        if (st1[j] <= np) std::snprintf(name, sizeof name, "patch-%08d.dat", st1[j]);
        else std::snprintf(name, sizeof name, "volume-%08d.dat", st1[j] - np);
        if (!open(fst[j], name)) return UCG_E_BADARG;
    }
    for (int k = 0; k < nobs; k++) {
        const char *nm = ucg_deck_point_name(deck, k);
        if (!open(fpt[k], std::string("opts-") + nm + ".dat")) return UCG_E_BADARG;
    }
    std::string line;
    std::fputs("#               time                 dt\n", ftime.f);
    line.clear();
    put_es(line, 0.0, 19, 12, 2);
    put_es(line, dt_next, 19, 12, 2);
    line += '\n';
    std::fputs(line.c_str(), ftime.f);
    if (opt->verbose) {
        std::printf("#       n               time                 dt       vMax\n");
        line = "000000000";
        put_es(line, 0.0, 19, 12, 2);
        put_es(line, dt_next, 19, 12, 2);
        std::printf("%s\n", line.c_str());
    }

    std::vector<double> rec((size_t)rlen * cap);
    long done = 0;
    double t = 0.0;
    int status = UCG_OK;
    while (done < opt->maximum_iterations) {
        const long todo = std::min(opt->chunk, opt->maximum_iterations - done);
        long steps = 0;
        status = ucg_run(c, info.interval, todo, &steps);
        long nrec = 0, lost = 0;
        if ((rc = ucg_records(c, rec.data(), cap, &nrec, &lost))) return rc;
        if (lost) return UCG_E_STATE;
        for (long r = 0; r < nrec; r++) {
            const double *q = &rec[(size_t)r * rlen];
            const long it = done + r + 1;   // the reference's iteration counter i
            line.clear();
            put_es(line, q[0], 19, 12, 2);
            put_es(line, q[1], 19, 12, 2);
            line += '\n';
            std::fputs(line.c_str(), ftime.f);
            for (int j = 0; j < nst; j++) {
                const int dgf = st1[j] <= np ? 7 : 12;
                const double *s = q + 4 + 24 * j;
                line.clear();
                put_es(line, q[0], 19, 12, 2);
                for (int m = 0; m < dgf; m++) put_es(line, s[m], 20, 12, 3);
                for (int m = 0; m < dgf; m++) put_es(line, s[12 + m], 20, 12, 3);
                line += '\n';
                std::fputs(line.c_str(), fst[j].f);
            }
            const double *dsp = q + 4 + 24 * nst;
            for (int k = 0; k < nobs; k++) {
                line.clear();
                put_es(line, q[0], 19, 12, 2);
                for (int m = 0; m < per_point; m++) put_es(line, dsp[per_point * k + m], 19, 12, 2);
                line += '\n';
                std::fputs(line.c_str(), fpt[k].f);
            }
            if (opt->verbose && it % 50 == 0) {
                char head[24];
                std::snprintf(head, sizeof head, "%09ld", it);
                line = head;
                put_es(line, q[0], 19, 12, 2);
                put_es(line, q[1], 19, 12, 2);
                put_es(line, q[2], 11, 4, 2);
                std::printf("%s\n", line.c_str());
            }
        }
        done += steps;
        long acc = 0, rej = 0;
        if ((rc = ucg_get_state(c, y.data(), &t, &dt_next, &acc, &rej))) return rc;
        if (status != UCG_OK || steps < todo || t >= info.interval) break;
    }
    if (opt->verbose) std::printf("%09ld time steps.\n", done);
    if (iterations) *iterations = done;
    if (time_out) *time_out = t;
    return status;
}
