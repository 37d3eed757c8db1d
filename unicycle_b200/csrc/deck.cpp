// Input decks of the reference's 3-D drivers, read on the host.
//
// The deck is the text the reference reads from standard input or from a file
// named on the command line: init() of fortran/3d/src/ratestate.f90:958-1739
// (UCG_DRIVER_RATESTATE) and of fortran/3d/src/viscouscycles.f90:1291-2069
// (UCG_DRIVER_VISCOUSCYCLES).  Sections, in order:
//
//   output directory                      (the whole line)
//   lambda mu
//   time interval
//   number of rectangular patches, then   i Vpl x1 x2 x3 length width strike dip rake
//     number of frictional rectangles (= the count), then   i mu0 sig a b L Vo damping
//   number of triangular patches, then    i Vpl i1 i2 i3 rake
//     number of vertices, then            i x1 x2 x3
//     number of frictional triangles (= the count), then the friction lines
//   [viscouscycles] number of strain volumes, then
//                      i e11 e12 e13 e22 e23 e33 x1 x2 x3 length width thickness strike dip
//     number of nonlinear Maxwell volumes (0 or the count), then   i Gm gammadot0m n Q R
//     number of thermal volumes (0 or the count), then             i rhoc To
//   number of observation patches, then   n i
//   [viscouscycles] number of observation volumes, then   n i
//   number of observation points, then    n name x1 x2 x3
//   number of perturbations, then one time per perturbation after the first
//
// Lines whose first non-blank character is '#' are skipped (getdata.f); so are
// blank lines.  Each data line is read list-directed: values separated by
// blanks or commas, '/' ends the line, r*v repeats v r times, D or d may mark
// the exponent, names may be quoted.  Angles are read in degrees and kept in
// radians.  The validation the reference performs while reading (indices in
// order, positive sizes, vertical volumes, counts that must match, increasing
// perturbation times) is kept, with the line number in the message instead of
// a STOP.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <vector>
#include "../../include/ucg.h"

struct ucg_deck {
    int driver = UCG_DRIVER_RATESTATE;
    std::string wdir;
    double lambda = 0, mu = 0, interval = 0;
    // rectangles (geometry) and triangles (connectivity, vertices)
    std::vector<double> rx, rL, rW, rstrike, rdip;
    std::vector<int> ti1, ti2, ti3;
    std::vector<double> tv;
    // per patch, rectangles then triangles
    std::vector<double> Vpl, rake, mu0, sig, a, b, L, Vo, damping;
    // strain volumes
    std::vector<double> vx, vL, vW, vT, vstrike, ebg;
    bool nonlinear = false, thermal = false;
    std::vector<double> nGm, ngd0, npow, nQm, nRm, rhoc, To;
    // observation states (1-based element indices, volumes after all patches),
    // observation points and perturbations
    std::vector<int> obs_state;
    std::vector<std::string> obs_name;
    std::vector<double> obs_x;
    std::vector<double> events;
};

namespace {

const double DEG2RAD = 0.017453292519943295;

struct DeckError {
    std::string msg;
};

class Reader {
public:
    explicit Reader(const std::string &text) : in_(text) {}

    // next data line (getdata.f), with its line number
    std::string line()
    {
        std::string s;
        while (std::getline(in_, s)) {
            lineno_++;
            if (!s.empty() && s.back() == '\r') s.pop_back();
            size_t i = s.find_first_not_of(" \t");
            if (i == std::string::npos || s[i] == '#') continue;
            return s;
        }
        fail("unexpected end of input");
        return s;
    }

    // list-directed tokens of the next data line
    std::vector<std::string> tokens()
    {
        const std::string s = line();
        std::vector<std::string> out;
        size_t i = 0;
        while (i < s.size()) {
            while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == ',')) i++;
            if (i >= s.size() || s[i] == '/') break;
            std::string tok;
            if (s[i] == '\'' || s[i] == '"') {
                const char q = s[i++];
                while (i < s.size() && s[i] != q) tok += s[i++];
                i++;
            } else {
                while (i < s.size() && s[i] != ' ' && s[i] != '\t' && s[i] != ',' && s[i] != '/') tok += s[i++];
            }
            // repeat count r*v
            const size_t star = tok.find('*');
            if (star != std::string::npos && star > 0 &&
                tok.find_first_not_of("0123456789") == star) {
                const long r = std::strtol(tok.substr(0, star).c_str(), nullptr, 10);
                for (long k = 0; k < r; k++) out.push_back(tok.substr(star + 1));
            } else {
                out.push_back(tok);
            }
        }
        return out;
    }

    [[noreturn]] void fail(const std::string &why) const
    {
        throw DeckError{"input deck line " + std::to_string(lineno_) + ": " + why};
    }

    double real(const std::vector<std::string> &t, size_t k) const
    {
        if (k >= t.size()) fail("missing value " + std::to_string(k + 1));
        std::string s = t[k];
        for (char &ch : s)
            if (ch == 'd' || ch == 'D') ch = 'e';
        char *end = nullptr;
        const double v = std::strtod(s.c_str(), &end);
        if (end == s.c_str() || *end != '\0') fail("not a number: '" + t[k] + "'");
        return v;
    }

    long integer(const std::vector<std::string> &t, size_t k) const
    {
        if (k >= t.size()) fail("missing value " + std::to_string(k + 1));
        char *end = nullptr;
        const long v = std::strtol(t[k].c_str(), &end, 10);
        if (end == t[k].c_str() || *end != '\0') fail("not an integer: '" + t[k] + "'");
        return v;
    }

    long count()
    {
        const auto t = tokens();
        const long n = integer(t, 0);
        if (n < 0) fail("negative count");
        return n;
    }

    void index(const std::vector<std::string> &t, long k) const
    {
        if (integer(t, 0) != k) fail("unexpected index (expected " + std::to_string(k) + ")");
    }

private:
    std::istringstream in_;
    long lineno_ = 0;
};

void read_friction(Reader &r, ucg_deck *d, long n, const char *what)
{
    if (r.count() != n) r.fail(std::string("all ") + what + " patches require frictional properties");
    for (long k = 1; k <= n; k++) {
        const auto t = r.tokens();
        r.index(t, k);
        d->mu0.push_back(r.real(t, 1));
        d->sig.push_back(r.real(t, 2));
        d->a.push_back(r.real(t, 3));
        d->b.push_back(r.real(t, 4));
        d->L.push_back(r.real(t, 5));
        d->Vo.push_back(r.real(t, 6));
        d->damping.push_back(r.real(t, 7));
    }
}

void parse(const std::string &text, ucg_deck *d)
{
    Reader r(text);
    // output directory (READ '(a)': the whole line)
    {
        std::string s = r.line();
        const size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
        d->wdir = s.substr(a, b - a + 1);
    }
    {
        const auto t = r.tokens();
        d->lambda = r.real(t, 0);
        d->mu = r.real(t, 1);
        if (0.0 > d->mu) r.fail("shear modulus must be positive");
        const double nu = d->lambda / 2.0 / (d->lambda + d->mu);
        if (-1.0 > nu) r.fail("Poisson's ratio must be greater than -1");
        if (0.5 < nu) r.fail("Poisson's ratio must be lower than 0.5");
    }
    {
        const auto t = r.tokens();
        d->interval = r.real(t, 0);
        if (d->interval <= 0.0) r.fail("simulation time must be positive");
    }
    // rectangular patches
    const long nr = r.count();
    if (nr > 0) {
        for (long k = 1; k <= nr; k++) {
            const auto t = r.tokens();
            r.index(t, k);
            d->Vpl.push_back(r.real(t, 1));
            for (int c = 0; c < 3; c++) d->rx.push_back(r.real(t, 2 + c));
            d->rL.push_back(r.real(t, 5));
            d->rW.push_back(r.real(t, 6));
            d->rstrike.push_back(r.real(t, 7) * DEG2RAD);
            d->rdip.push_back(r.real(t, 8) * DEG2RAD);
            d->rake.push_back(r.real(t, 9) * DEG2RAD);
            if (std::fmax(d->rL.back(), d->rW.back()) <= 0.0) r.fail("patch length and width must be positive");
        }
        read_friction(r, d, nr, "rectangular");
    }
    // triangular patches
    const long nt = r.count();
    if (nt > 0) {
        std::vector<double> tVpl, trake;
        long maxv = -1;
        for (long k = 1; k <= nt; k++) {
            const auto t = r.tokens();
            r.index(t, k);
            tVpl.push_back(r.real(t, 1));
            const long i1 = r.integer(t, 2), i2 = r.integer(t, 3), i3 = r.integer(t, 4);
            trake.push_back(r.real(t, 5) * DEG2RAD);
            if (i1 < 1 || i2 < 1 || i3 < 1) r.fail("vertex indices must be positive");
            maxv = std::max(maxv, std::max(i1, std::max(i2, i3)));
            d->ti1.push_back((int)i1);
            d->ti2.push_back((int)i2);
            d->ti3.push_back((int)i3);
        }
        const long nve = r.count();
        if (maxv > nve) r.fail("not enough vertices");
        for (long k = 1; k <= nve; k++) {
            const auto t = r.tokens();
            r.index(t, k);
            for (int c = 0; c < 3; c++) d->tv.push_back(r.real(t, 1 + c));
        }
        d->Vpl.insert(d->Vpl.end(), tVpl.begin(), tVpl.end());
        d->rake.insert(d->rake.end(), trake.begin(), trake.end());
        read_friction(r, d, nt, "triangular");
    }
    const long np = nr + nt;
    long nv = 0;
    if (d->driver == UCG_DRIVER_VISCOUSCYCLES) {
        nv = r.count();
        if (nv > 0) {
            for (long k = 1; k <= nv; k++) {
                const auto t = r.tokens();
                r.index(t, k);
                for (int c = 0; c < 6; c++) d->ebg.push_back(r.real(t, 1 + c));
                for (int c = 0; c < 3; c++) d->vx.push_back(r.real(t, 7 + c));
                d->vL.push_back(r.real(t, 10));
                d->vW.push_back(r.real(t, 11));
                d->vT.push_back(r.real(t, 12));
                d->vstrike.push_back(r.real(t, 13) * DEG2RAD);
                if (90.0 != r.real(t, 14)) r.fail("strain volume must be vertical (dip=90)");
                if (0.0 > d->vx.back()) r.fail("depth must be positive");
                if (std::fmax(d->vL.back(), std::fmax(d->vW.back(), d->vT.back())) <= 0.0)
                    r.fail("strain volume dimension must be positive");
            }
            const long nn = r.count();
            if (nn != 0) {
                if (nn != nv) r.fail("nonlinear Maxwell properties are for none or all strain volumes");
                d->nonlinear = true;
                for (long k = 1; k <= nv; k++) {
                    const auto t = r.tokens();
                    r.index(t, k);
                    d->nGm.push_back(r.real(t, 1));
                    d->ngd0.push_back(r.real(t, 2));
                    d->npow.push_back(r.real(t, 3));
                    d->nQm.push_back(r.real(t, 4));
                    d->nRm.push_back(r.real(t, 5));
                    if (0.0 >= d->nGm.back()) r.fail("Gm must be positive");
                    if (0.0 >= d->nRm.back()) r.fail("R must be positive");
                }
            }
            const long nth = r.count();
            if (nth != 0) {
                if (nth != nv) r.fail("thermal properties are for none or all strain volumes");
                d->thermal = true;
                for (long k = 1; k <= nv; k++) {
                    const auto t = r.tokens();
                    r.index(t, k);
                    d->rhoc.push_back(r.real(t, 1));
                    d->To.push_back(r.real(t, 2));
                    if (0.0 >= d->To.back()) r.fail("To must be positive");
                }
            }
        }
    }
    // observation patches (and volumes)
    const long nop = r.count();
    for (long k = 1; k <= nop; k++) {
        const auto t = r.tokens();
        r.index(t, k);
        const long e = r.integer(t, 1);
        if (e < 1 || e > (d->driver == UCG_DRIVER_VISCOUSCYCLES ? np : np)) r.fail("observation patch out of range");
        d->obs_state.push_back((int)e);
    }
    if (d->driver == UCG_DRIVER_VISCOUSCYCLES) {
        const long nov = r.count();
        for (long k = 1; k <= nov; k++) {
            const auto t = r.tokens();
            r.index(t, k);
            const long e = r.integer(t, 1);
            if (e < 1 || e > nv) r.fail("observation volume out of range");
            d->obs_state.push_back((int)(e + np));
        }
    }
    // observation points
    const long nobs = r.count();
    for (long k = 1; k <= nobs; k++) {
        const auto t = r.tokens();
        r.index(t, k);
        if (t.size() < 2) r.fail("missing observation point name");
        d->obs_name.push_back(t[1].substr(0, 10));   // CHARACTER(LEN=10)
        for (int c = 0; c < 3; c++) d->obs_x.push_back(r.real(t, 2 + c));
    }
    // perturbations: the first at t = 0, then one time per line, increasing
    const long ne = r.count();
    for (long k = 1; k <= ne; k++) {
        if (k == 1) {
            d->events.push_back(0.0);
            continue;
        }
        const auto t = r.tokens();
        const double tk = r.real(t, 0);
        if (tk <= d->events.back()) r.fail("timing of perturbations must increase");
        d->events.push_back(tk);
    }
    if ((np == 0 && nv == 0) || d->interval <= 0.0) r.fail("nothing to do");
}

void put_err(char *err, long len, const std::string &msg)
{
    if (err && len > 0) {
        std::strncpy(err, msg.c_str(), (size_t)len - 1);
        err[len - 1] = '\0';
    }
}

template <class T>
long copy_out(const std::vector<T> &v, T *out, long max)
{
    if (out) {
        const long k = std::min<long>((long)v.size(), max);
        for (long i = 0; i < k; i++) out[i] = v[i];
    }
    return (long)v.size();
}

}  // namespace

extern "C" {

int ucg_deck_parse(const char *text, int driver, ucg_deck **deck, char *err, long err_len)
{
    if (!text || !deck) return UCG_E_BADARG;
    *deck = nullptr;
    if (driver != UCG_DRIVER_RATESTATE && driver != UCG_DRIVER_VISCOUSCYCLES) return UCG_E_BADARG;
    ucg_deck *d = new (std::nothrow) ucg_deck();
    if (!d) return UCG_E_OOM;
    d->driver = driver;
    try {
        parse(text, d);
    } catch (const DeckError &e) {
        put_err(err, err_len, e.msg);
        delete d;
        return UCG_E_BADARG;
    } catch (const std::bad_alloc &) {
        delete d;
        return UCG_E_OOM;
    }
    put_err(err, err_len, "");
    *deck = d;
    return UCG_OK;
}

int ucg_deck_read(const char *path, int driver, ucg_deck **deck, char *err, long err_len)
{
    if (!path || !deck) return UCG_E_BADARG;
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        put_err(err, err_len, std::string("unable to access ") + path);
        return UCG_E_BADARG;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    return ucg_deck_parse(ss.str().c_str(), driver, deck, err, err_len);
}

void ucg_deck_free(ucg_deck *d) { delete d; }

int ucg_deck_summary(const ucg_deck *d, ucg_deck_info *s)
{
    if (!d || !s) return UCG_E_BADARG;
    s->driver = d->driver;
    s->lambda = d->lambda;
    s->mu = d->mu;
    s->interval = d->interval;
    s->n_rect = (int)d->rL.size();
    s->n_tri = (int)d->ti1.size();
    s->n_vertex = (int)(d->tv.size() / 3);
    s->n_vol = (int)d->vL.size();
    s->nonlinear_maxwell = d->nonlinear ? 1 : 0;
    s->thermal = d->thermal ? 1 : 0;
    s->n_obs_state = (int)d->obs_state.size();
    s->n_obs_point = (int)d->obs_name.size();
    s->n_events = (int)d->events.size();
    return UCG_OK;
}

const char *ucg_deck_wdir(const ucg_deck *d) { return d ? d->wdir.c_str() : ""; }

const char *ucg_deck_point_name(const ucg_deck *d, int k)
{
    if (!d || k < 0 || k >= (int)d->obs_name.size()) return nullptr;
    return d->obs_name[k].c_str();
}

long ucg_deck_get(const ucg_deck *d, const char *field, double *out, long max)
{
    if (!d || !field) return UCG_E_BADARG;
    struct F {
        const char *name;
        const std::vector<double> *v;
    } table[] = {
        {"rect.x", &d->rx}, {"rect.length", &d->rL}, {"rect.width", &d->rW}, {"rect.strike", &d->rstrike},
        {"rect.dip", &d->rdip}, {"tri.vertices", &d->tv}, {"patch.Vpl", &d->Vpl}, {"patch.rake", &d->rake},
        {"patch.mu0", &d->mu0}, {"patch.sig", &d->sig}, {"patch.a", &d->a}, {"patch.b", &d->b},
        {"patch.L", &d->L}, {"patch.Vo", &d->Vo}, {"patch.damping", &d->damping}, {"vol.x", &d->vx},
        {"vol.length", &d->vL}, {"vol.width", &d->vW}, {"vol.thickness", &d->vT}, {"vol.strike", &d->vstrike},
        {"vol.e_bg", &d->ebg}, {"vol.Gm", &d->nGm}, {"vol.gammadot0m", &d->ngd0}, {"vol.npowerm", &d->npow},
        {"vol.Q", &d->nQm}, {"vol.R", &d->nRm}, {"vol.rhoc", &d->rhoc}, {"vol.To", &d->To},
        {"obs.x", &d->obs_x}, {"events.time", &d->events},
    };
    for (const F &f : table)
        if (!std::strcmp(field, f.name)) return copy_out(*f.v, out, max);
    return UCG_E_BADARG;
}

long ucg_deck_get_int(const ucg_deck *d, const char *field, int *out, long max)
{
    if (!d || !field) return UCG_E_BADARG;
    if (!std::strcmp(field, "tri.i1")) return copy_out(d->ti1, out, max);
    if (!std::strcmp(field, "tri.i2")) return copy_out(d->ti2, out, max);
    if (!std::strcmp(field, "tri.i3")) return copy_out(d->ti3, out, max);
    if (!std::strcmp(field, "obs.state")) return copy_out(d->obs_state, out, max);
    return UCG_E_BADARG;
}

int ucg_deck_apply(const ucg_deck *d, ucg_ctx *c)
{
    if (!d || !c) return UCG_E_BADARG;
    const int nr = (int)d->rL.size(), nt = (int)d->ti1.size(), nv = (int)d->vL.size();
    int rc;
    if ((rc = ucg_set_rectangles(c, nr, d->rx.data(), d->rL.data(), d->rW.data(), d->rstrike.data(),
                                 d->rdip.data())))
        return rc;
    if ((rc = ucg_set_triangles(c, nt, d->ti1.data(), d->ti2.data(), d->ti3.data(), (int)(d->tv.size() / 3),
                                d->tv.data())))
        return rc;
    if ((rc = ucg_set_volumes(c, nv, d->vx.data(), d->vL.data(), d->vT.data(), d->vW.data(), d->vstrike.data())))
        return rc;
    if (nr + nt > 0 &&
        (rc = ucg_set_friction(c, d->Vpl.data(), d->rake.data(), d->mu0.data(), d->sig.data(), d->a.data(),
                               d->b.data(), d->L.data(), d->Vo.data(), d->damping.data())))
        return rc;
    if (nv > 0) {
        // without nonlinear Maxwell properties the reference's fields stay zero
        std::vector<double> z(nv, 0.0);
        const double *g = d->nonlinear ? d->ngd0.data() : z.data();
        const double *p = d->nonlinear ? d->npow.data() : z.data();
        if ((rc = ucg_set_rheology(c, d->ebg.data(), g, p, d->nonlinear ? 1 : 0))) return rc;
    }
    if (!d->obs_name.empty() &&
        (rc = ucg_set_observation_points(c, (int)d->obs_name.size(), d->obs_x.data())))
        return rc;
    return UCG_OK;
}

int ucg_deck_create(const ucg_deck *d, int device, ucg_ctx **ctx)
{
    if (!d || !ctx) return UCG_E_BADARG;
    int rc = ucg_create(ctx, device, d->mu, d->lambda, d->driver);
    if (rc) return rc;
    if ((rc = ucg_deck_apply(d, *ctx))) {
        ucg_destroy(*ctx);
        *ctx = nullptr;
    }
    return rc;
}

int ucg_deck_init_state(const ucg_deck *d, ucg_ctx *c, double *y)
{
    if (!d || !c || !y) return UCG_E_BADARG;
    const size_t nv = d->vL.size();
    std::vector<double> z(nv, 0.0), one(nv, 1.0);
    const double *Gm = d->nonlinear ? d->nGm.data() : z.data();
    const double *Q = d->nonlinear ? d->nQm.data() : z.data();
    const double *R = d->nonlinear ? d->nRm.data() : one.data();
    const double *To = d->thermal ? d->To.data() : one.data();
    return ucg_init_state(c, y, nv ? Gm : nullptr, nv ? Q : nullptr, nv ? R : nullptr, nv ? To : nullptr);
}

}  // extern "C"
