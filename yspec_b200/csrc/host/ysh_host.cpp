// ysh_host.cpp -- C++ host of the `yspec input.in` program.
//
// Mirrors the reference's Fortran host above the ysg_* boundary:
//   parameter file      yspec.f90:79-139, module_util.f90:301-355
//   model file          module_model.f90:175-383, module_spline.f90:40-73,426-449
//   event setup         yspec.f90:144-215, module_function.f90:317-390 (delaz),
//                       module_fourier.f90:362-397 (fcal),
//                       module_model.f90:537-576 (find_radius_index)
//   writer              yspec.f90:488-503, module_util.f90:428-444
// Formats, stop conditions and the single-precision quirks of these
// routines are kept; the numerical kernels run on the GPU through ysg_*.
#include "yspec_host.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <atomic>
#include <chrono>
#include <map>
#include <string>
#include <thread>
#include <vector>

namespace {

// nrtype.f90:18-27: pi_d, twopi_d are single-precision literals.
const double kPi = (double)3.14159265358979323846f;
const double kTwoPi = (double)6.28318530717958647692f;
const double kBigG = 6.6723e-11;

// ---------------------------------------------------------------------------
// Fortran list-directed input: a read statement starts on a fresh record and
// consumes records until its items are satisfied; blanks and commas
// separate values, a slash ends the read, the rest of the record is dropped.
// ---------------------------------------------------------------------------
class Records {
  public:
    explicit Records(const char* path) : in_(path) {}
    bool ok() const { return in_.good() || in_.eof(); }
    bool open() const { return in_.is_open(); }
    bool skip(int n)
    {
        std::string line;
        for (int i = 0; i < n; i++)
            if (!std::getline(in_, line)) return false;
        return true;
    }
    bool values(size_t k, std::vector<std::string>& out)
    {
        out.clear();
        std::string line;
        while (out.size() < k) {
            if (!std::getline(in_, line)) return false;
            size_t i = 0, n = line.size();
            while (i < n && out.size() < k) {
                while (i < n && (std::isspace((unsigned char)line[i]) || line[i] == ',')) i++;
                if (i >= n) break;
                if (line[i] == '/') return out.size() == k;
                std::string tok;
                if (line[i] == '\'' || line[i] == '"') {
                    char q = line[i++];
                    while (i < n && line[i] != q) tok += line[i++];
                    if (i < n) i++;
                } else {
                    while (i < n && !std::isspace((unsigned char)line[i]) && line[i] != ',' &&
                           line[i] != '/')
                        tok += line[i++];
                }
                out.push_back(tok);
            }
        }
        return true;
    }

  private:
    std::ifstream in_;
};

double to_real(std::string s)
{
    for (char& ch : s)
        if (ch == 'd' || ch == 'D') ch = 'e';
    return std::strtod(s.c_str(), nullptr);
}

int to_int(const std::string& s) { return (int)std::strtol(s.c_str(), nullptr, 10); }

// ---------------------------------------------------------------------------
// Natural cubic spline per layer (module_spline.f90:40-73): second
// derivatives from the tridiagonal system h_{i-1} y2_{i-1} +
// 2(h_{i-1}+h_i) y2_i + h_i y2_{i+1} = 6 (dy_i/h_i - dy_{i-1}/h_{i-1}) with
// y2 = 0 at both ends, solved by forward elimination and back substitution
// in the order of tridag_ser (module_spline.f90:426-449).
// ---------------------------------------------------------------------------
void natural_spline(const double* x, const double* y, int n, double* y2)
{
    if (n <= 0) return;
    std::vector<double> h(n, 0.0), rhs(n, 0.0), diag(n, 1.0), sub(n, 0.0), sup(n, 0.0);
    for (int i = 0; i + 1 < n; i++) h[i] = x[i + 1] - x[i];
    std::vector<double> slope(n, 0.0);
    for (int i = 0; i + 1 < n; i++) slope[i] = 6.0 * ((y[i + 1] - y[i]) / h[i]);
    for (int i = 1; i + 1 < n; i++) {
        rhs[i] = slope[i] - slope[i - 1];
        sub[i] = h[i - 1];
        diag[i] = 2.0 * (h[i] + sub[i]);
        sup[i] = h[i];
    }
    // natural ends: first and last rows are y2 = 0
    rhs[0] = 0.0;
    sup[0] = 0.0;
    rhs[n - 1] = 0.0;
    sub[n - 1] = 0.0;
    std::vector<double> gam(n, 0.0);
    double bet = diag[0];
    y2[0] = rhs[0] / bet;
    for (int j = 1; j < n; j++) {
        gam[j] = sup[j - 1] / bet;
        bet = diag[j] - sub[j] * gam[j];
        y2[j] = (rhs[j] - sub[j] * y2[j - 1]) / bet;
    }
    for (int j = n - 2; j >= 0; j--) y2[j] = y2[j] - gam[j + 1] * y2[j + 1];
}

// Cubic spline value on interval [lo, lo+1] (module_spline.f90:262-283).
double spline_eval(const std::vector<double>& xa, const std::vector<double>& ya,
                   const std::vector<double>& y2, double x, int lo)
{
    double h = xa[lo + 1] - xa[lo];
    if (h == 0.0) return ya[lo];
    double a = (xa[lo + 1] - x) / h, b = (x - xa[lo]) / h;
    return a * ya[lo] + b * ya[lo + 1] +
           ((a * a * a - a) * y2[lo] + (b * b * b - b) * y2[lo + 1]) * (h * h) / 6.0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Model (module_model.f90:175-383).  Arrays are 0-based here: knot k of the
// reference is index k-1.
// ---------------------------------------------------------------------------
struct ysh_model {
    int nknot = 0, nic = 0, noc = 0, nsl = 0, nlayer = 0;
    bool ifanis = false, ocean = false, fic = false;
    double tref = 0.0;
    std::vector<int> lay_lo, lay_hi;     // 0-based inclusive knot ranges
    std::vector<double> r, rho, acon, ccon, fcon, lcon, ncon, kappa, mu, lambda;
    std::vector<double> qkappa, qmu, grav, beta, alpha, rat, xlam, xa2;
    std::vector<double> cs[13];          // spline second derivatives, ysg order
    const std::vector<double>& val(int p) const
    {
        const std::vector<double>* v[13] = {&rho, &acon, &ccon, &fcon, &lcon, &ncon, &kappa,
                                            &mu, &qkappa, &qmu, &grav, &xlam, &xa2};
        return *v[p];
    }
    void spline_layers(const std::vector<double>& y, std::vector<double>& y2) const
    {
        y2.assign(nknot, 0.0);
        for (int L = 0; L < nlayer; L++) {
            int lo = lay_lo[L], n = lay_hi[L] - lay_lo[L] + 1;
            natural_spline(&r[lo], &y[lo], n, &y2[lo]);
        }
    }
};

extern "C" {

void ysh_norms_get(ysh_norms* n)
{
    // module_model.f90:474-492
    n->r_norm = 6.371e+6;
    n->rho_norm = 5.515e+3;
    n->vel_norm = n->r_norm * std::sqrt(kPi * kBigG * n->rho_norm);
    n->acl_norm = kPi * kBigG * n->rho_norm * n->r_norm;
    n->fre_norm = n->vel_norm / n->r_norm;
    n->t_norm = 1.0 / n->fre_norm;
    n->con_norm = n->vel_norm * n->vel_norm * n->rho_norm;
    n->grav_norm = kPi * kBigG;
    double r2 = n->r_norm * n->r_norm;
    n->moment_norm = (r2 * r2 * n->r_norm) * (n->rho_norm * n->rho_norm) * n->grav_norm;
    n->pot_norm = n->acl_norm * n->r_norm;
    n->pibigg = kPi * kBigG / n->grav_norm;
}

int ysh_read_params(const char* path, ysh_params* p)
{
    std::memset(p, 0, sizeof *p);
    Records rec(path);
    if (!rec.open()) return YSH_ERR_PARAM_FILE;
    std::vector<std::string> v;
    auto str = [&](char* dst, int skip) {
        if (!rec.skip(skip) || !rec.values(1, v)) return false;
        std::snprintf(dst, 256, "%s", v[0].c_str());
        return true;
    };
    auto num = [&](double* dst, int skip) {
        if (!rec.skip(skip) || !rec.values(1, v)) return false;
        *dst = to_real(v[0]);
        return true;
    };
    auto inum = [&](int* dst, int skip) {
        if (!rec.skip(skip) || !rec.values(1, v)) return false;
        *dst = to_int(v[0]);
        return true;
    };
    bool ok = str(p->pref_out, 4) && str(p->model_file, 2) && inum(&p->ats, 2) &&
              inum(&p->grav, 2) && inum(&p->out, 2) && inum(&p->cor, 2) && inum(&p->lmin, 2) &&
              inum(&p->lmax, 2) && num(&p->f1, 2) && num(&p->f2, 2) && num(&p->tout, 2) &&
              num(&p->dt, 2) && num(&p->f11, 2) && num(&p->f12, 2) && num(&p->f21, 2) &&
              num(&p->f22, 2) && num(&p->depth_s, 2) && num(&p->lat_s, 2) && num(&p->lon_s, 2);
    for (int i = 0; ok && i < 6; i++) ok = num(&p->mm[i], 2);
    ok = ok && num(&p->depth_r, 2) && inum(&p->nr, 2);
    if (ok && p->nr > 0) {
        ok = rec.skip(2);
        p->lat_r = (double*)std::calloc((size_t)p->nr, sizeof(double));
        p->lon_r = (double*)std::calloc((size_t)p->nr, sizeof(double));
        for (int i = 0; ok && i < p->nr; i++) {
            ok = rec.values(2, v);
            if (ok) {
                p->lat_r[i] = to_real(v[0]);
                p->lon_r[i] = to_real(v[1]);
            }
        }
    }
    if (!ok) {
        ysh_free_params(p);
        return YSH_ERR_PARAM_READ;
    }
    return YSH_OK;
}

void ysh_free_params(ysh_params* p)
{
    std::free(p->lat_r);
    std::free(p->lon_r);
    p->lat_r = p->lon_r = nullptr;
}

int ysh_read_model(const char* path, ysh_model** out)
{
    *out = nullptr;
    Records rec(path);
    if (!rec.open()) return YSH_ERR_MODEL_FILE;
    ysh_norms nm;
    ysh_norms_get(&nm);
    auto m = std::make_unique<ysh_model>();
    std::vector<std::string> v;
    if (!rec.values(1, v)) return YSH_ERR_MODEL_READ;            // title
    if (!rec.values(2, v)) return YSH_ERR_MODEL_READ;
    m->ifanis = to_int(v[0]) == 1;
    m->tref = (kTwoPi / to_real(v[1])) / nm.fre_norm;            // :195-197
    if (!rec.values(3, v)) return YSH_ERR_MODEL_READ;
    const int n = to_int(v[0]);
    m->nknot = n;
    m->nic = to_int(v[1]);
    m->noc = to_int(v[2]);
    if (n < 2) return YSH_ERR_MODEL_READ;
    for (auto* a : {&m->r, &m->rho, &m->acon, &m->ccon, &m->fcon, &m->lcon, &m->ncon, &m->kappa,
                    &m->mu, &m->lambda, &m->qkappa, &m->qmu, &m->grav, &m->beta, &m->alpha,
                    &m->rat, &m->xlam, &m->xa2})
        a->assign(n, 0.0);
    const size_t want = m->ifanis ? 9 : 6;
    for (int i = 0; i < n; i++) {                                // :209-222
        if (!rec.values(want, v)) return YSH_ERR_MODEL_READ;
        m->r[i] = to_real(v[0]);
        m->rho[i] = to_real(v[1]);
        m->ccon[i] = to_real(v[2]);
        m->lcon[i] = to_real(v[3]);
        m->qkappa[i] = to_real(v[4]);
        m->qmu[i] = to_real(v[5]);
        if (m->ifanis) {
            m->acon[i] = to_real(v[6]);
            m->ncon[i] = to_real(v[7]);
            m->fcon[i] = to_real(v[8]);
        } else {
            m->acon[i] = m->ccon[i];
            m->ncon[i] = m->lcon[i];
            m->fcon[i] = 1.0;
        }
    }
    // ocean and fluid inner core, :227-248 (nsl stored 1-based)
    m->ocean = m->lcon[n - 1] == 0.0;
    m->nsl = n;
    if (m->ocean) {
        m->nsl = 0;
        for (int i = n - 2; i >= 0; i--)
            if (m->lcon[i] > 0.0) { m->nsl = i + 1; break; }
    }
    m->fic = m->lcon[0] == 0.0;
    // normalisation and moduli, :253-290
    for (int i = 0; i < n; i++) {
        double rho = m->rho[i] / nm.rho_norm;
        double va = m->acon[i] / nm.vel_norm, vc = m->ccon[i] / nm.vel_norm;
        double vl = m->lcon[i] / nm.vel_norm, vn = m->ncon[i] / nm.vel_norm;
        m->r[i] = m->r[i] / nm.r_norm;
        m->rho[i] = rho;
        m->acon[i] = rho * (va * va);
        m->ccon[i] = rho * (vc * vc);
        m->lcon[i] = rho * (vl * vl);
        m->ncon[i] = rho * (vn * vn);
        m->fcon[i] = (m->acon[i] - 2.0 * m->lcon[i]) * m->fcon[i];
        m->kappa[i] = (m->ccon[i] + 4.0 * m->acon[i] - 4.0 * m->ncon[i] + 4.0 * m->fcon[i]) / 9.0;
        m->mu[i] = (m->ccon[i] + m->acon[i] + 6.0 * m->lcon[i] + 5.0 * m->ncon[i] -
                    2.0 * m->fcon[i]) / 15.0;
        m->lambda[i] = m->kappa[i] - 2.0 * m->mu[i] / 3.0;
        m->beta[i] = std::sqrt(m->mu[i] / rho);
        m->alpha[i] = std::sqrt((m->kappa[i] + 1.3333333333 * m->mu[i]) / rho);
        if (m->qkappa[i] > 0.0) m->qkappa[i] = 1.0 / m->qkappa[i];
        if (m->qmu[i] > 0.0) m->qmu[i] = 1.0 / m->qmu[i];
        double rat = 4.0 * m->mu[i] / (3.0 * (m->lambda[i] + 2.0 * m->mu[i]));
        m->rat[i] = rat;
        m->xlam[i] = ((1.0 - rat) * m->qkappa[i] - 0.5 * rat * m->qmu[i]) / (1.0 - 1.5 * rat);
        m->xa2[i] = (1.0 - rat) * m->qkappa[i] + rat * m->qmu[i];
    }
    // layers split at repeated radii, :294-308
    m->lay_lo.push_back(0);
    for (int i = 1; i < n; i++)
        if (m->r[i] == m->r[i - 1]) {
            m->lay_hi.push_back(i - 1);
            m->lay_lo.push_back(i);
        }
    m->lay_hi.push_back(n - 1);
    m->nlayer = (int)m->lay_lo.size();
    // splines, :312-352 (ysg parameter order; grav after gravity below)
    for (int p = 0; p < 13; p++)
        if (p != 10) m->spline_layers(m->val(p), m->cs[p]);
    // gravity: 5-point Gauss-Legendre (constants of gauslv, :507-535) on a
    // spline of r^2 rho, then g = 4 int / r^2, :356-371
    {
        std::vector<double> intg(n), q2;
        for (int i = 0; i < n; i++) intg[i] = (m->r[i] * m->r[i]) * m->rho[i];
        m->spline_layers(intg, q2);
        const double w1 = .478628670499366, w2 = .236926885056189, w0 = .568888888888889;
        const double x1 = .538469310105683, x2 = .906179845938664;
        double fint = 0.0;
        m->grav[0] = 0.0;
        for (int i = 0; i + 1 < n; i++) {
            double a = m->r[i], b = m->r[i + 1];
            double mid = 0.5 * (b + a), half = 0.5 * (b - a);
            double sum = w0 * spline_eval(m->r, intg, q2, mid, i);
            double t = x1 * half;
            sum = sum + w1 * (spline_eval(m->r, intg, q2, mid + t, i) +
                              spline_eval(m->r, intg, q2, mid - t, i));
            t = x2 * half;
            sum = sum + w2 * (spline_eval(m->r, intg, q2, mid + t, i) +
                              spline_eval(m->r, intg, q2, mid - t, i));
            fint = fint + half * sum;
            m->grav[i + 1] = fint;
        }
        for (int i = 0; i < n; i++)
            if (m->r[i] > 0.0) m->grav[i] = (4.0 * m->grav[i]) / (m->r[i] * m->r[i]);
        m->spline_layers(m->grav, m->cs[10]);
    }
    *out = m.release();
    return YSH_OK;
}

void ysh_model_view(const ysh_model* m, ysg_model* v)
{
    std::memset(v, 0, sizeof *v);
    ysh_norms nm;
    ysh_norms_get(&nm);
    v->nknot = m->nknot;
    v->nic = m->nic;
    v->noc = m->noc;
    v->nsl = m->nsl;
    v->ocean = m->ocean;
    v->fic = m->fic;
    v->tref = m->tref;
    v->pibigg = nm.pibigg;
    v->fre_norm = nm.fre_norm;
    v->r = m->r.data();
    for (int p = 0; p < 13; p++) {
        v->val[p] = m->val(p).data();
        v->cs[p] = m->cs[p].data();
    }
    v->alpha = m->alpha.data();
    v->beta = m->beta.data();
}

int ysh_model_nknot(const ysh_model* m) { return m->nknot; }

const double* ysh_model_array(const ysh_model* m, const char* name)
{
    static const char* names[13] = {"rho", "acon", "ccon", "fcon", "lcon", "ncon", "kappa",
                                    "mu", "qkappa", "qmu", "grav", "xlam", "xa2"};
    std::string s(name);
    if (s == "r") return m->r.data();
    if (s == "alpha") return m->alpha.data();
    if (s == "beta") return m->beta.data();
    for (int p = 0; p < 13; p++) {
        if (s == names[p]) return m->val(p).data();
        if (s == std::string(names[p]) + "_cs") return m->cs[p].data();
    }
    return nullptr;
}

void ysh_free_model(ysh_model* m) { delete m; }

}  // extern "C"

namespace {

// module_function.f90:317-390 delaz (called with the receiver as "epicentre")
void delaz(double eplati, double eplong, double stlati, double stlong, double* delta,
           double* azep, double* azst)
{
    const double geoco = 0.993277, hpi = 0.5 * kPi, rad = 0.0174533;
    double eplat = eplati == -90.0 ? -89.98 : eplati;
    double stlat = stlati == -90.0 ? -89.98 : stlati;
    if (eplat == stlat && eplong == stlong) {
        *delta = *azep = *azst = 0.0;
        return;
    }
    double el = hpi - std::atan(geoco * std::tan(eplat * rad));
    double stl = hpi - std::atan(geoco * std::tan(stlat * rad));
    double elon = eplong * rad, slon = stlong * rad;
    double as = std::cos(stl), bs = std::sin(stl), cs = std::cos(slon), ds = std::sin(slon);
    double a = std::cos(el), b = std::sin(el), c = std::cos(elon), d = std::sin(elon);
    double cdel = a * as + b * bs * (c * cs + d * ds);
    if (std::fabs(cdel) > 1.0) cdel = std::copysign(1.0, cdel);
    double delt = std::acos(cdel);
    *delta = delt;
    double sdel = std::sin(delt);
    double caze = (as - a * cdel) / (sdel * b);
    if (std::fabs(caze) > 1.0) caze = std::copysign(1.0, caze);
    double aze = std::acos(caze);
    double cazs = 0.0;
    if (bs > 0.0) cazs = (a - as * cdel) / (bs * sdel);
    if (bs == 0.0) cazs = std::copysign(1.0, cazs);
    if (std::fabs(cazs) > 1.0) cazs = std::copysign(1.0, cazs);
    double azs = std::acos(cazs);
    double dif = ds * c - cs * d;
    if (dif < 0.0) aze = kTwoPi - aze;
    *azep = aze;
    if (dif > 0.0) azs = kTwoPi - azs;
    *azst = azs;
}

// module_model.f90:537-576 with up = -1
int radius_index(const ysh_model* m, double rr)
{
    if (rr < 0.0 || rr > 1.0) return 0;
    for (int i = 0; i + 1 < m->nknot; i++) {
        if (rr == m->r[i] && rr == m->r[i + 1]) return i + 1;
        if (rr > m->r[i] && rr <= m->r[i + 1]) return i + 1;
    }
    return 0;
}

// gfortran E15.6 field: [-]0.dddddd E+ee right-justified in 15 columns
void e15_6(double x, char* field)
{
    char t[40], body[32], dig[8];
    double ax = std::fabs(x);
    int e10 = 0;
    if (ax == 0.0) {
        std::memcpy(dig, "000000", 7);
    } else {
        std::snprintf(t, sizeof t, "%.5e", ax);
        dig[0] = t[0];
        std::memcpy(dig + 1, t + 2, 5);
        dig[6] = 0;
        e10 = std::atoi(std::strchr(t, 'e') + 1) + 1;
    }
    int ae = std::abs(e10);
    const char* sg = std::signbit(x) ? "-" : "";
    if (ae <= 99)
        std::snprintf(body, sizeof body, "%s0.%sE%c%02d", sg, dig, e10 < 0 ? '-' : '+', ae);
    else
        std::snprintf(body, sizeof body, "%s0.%s%c%03d", sg, dig, e10 < 0 ? '-' : '+', ae);
    std::snprintf(field, 16, "%15.15s", body);
}

// Powers of ten that a double holds exactly.
const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                           1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// The six significant digits D (100000 <= D < 1000000) and the exponent
// e10 of an E15.6 field for a finite ax > 0, formed without snprintf:
// y = ax 10^(5 - E) with E = floor(log10 ax) takes one correctly rounded
// product or quotient by an exact power of ten, so |y - exact| <= 1.2e-10;
// D = round(y) is then certain unless the exact value lies within 1e-6 of
// a rounding boundary (a half-integer, 1e5 or 1e6), or 10^(5 - E) is not
// exact.  Those cases return false and take the snprintf path, so the
// field is the same text either way.
bool e15_digits(double ax, int* digits, int* e10)
{
    int E = (int)std::floor(std::log10(ax));
    double y = 0.0;
    for (int pass = 0; pass < 3; pass++) {
        const int k = 5 - E;
        if (k >= 0 && k <= 22) y = ax * kPow10[k];
        else if (k < 0 && k >= -22) y = ax / kPow10[-k];
        else return false;
        if (y < 1e5) E--;
        else if (y >= 1e6) E++;
        else break;
        if (pass == 2) return false;
    }
    if (y < 1e5 + 1e-4 || y > 1e6 - 0.5 - 1e-6) return false;
    const double fl = std::floor(y), fr = y - fl;
    if (std::fabs(fr - 0.5) < 1e-6) return false;
    int d = (int)fl + (fr > 0.5 ? 1 : 0);
    *digits = d;
    *e10 = E + 1;
    return true;
}

// e15_6 with the digits formed by e15_digits where it can.
void e15_6_fast(double x, char* field)
{
    const double ax = std::fabs(x);
    int d = 0, e10 = 0;
    if (ax == 0.0) {
        d = -1;                                        // all-zero digits, exponent 0
    } else if (!(std::isfinite(ax) && e15_digits(ax, &d, &e10))) {
        e15_6(x, field);
        return;
    }
    char body[16];
    int n = 0;
    if (std::signbit(x)) body[n++] = '-';
    body[n++] = '0';
    body[n++] = '.';
    if (d < 0) {
        for (int i = 0; i < 6; i++) body[n++] = '0';
    } else {
        for (int i = 5; i >= 0; i--) {
            body[n + i] = (char)('0' + d % 10);
            d /= 10;
        }
        n += 6;
    }
    const int ae = e10 < 0 ? -e10 : e10;
    if (ae <= 99) {
        body[n++] = 'E';
        body[n++] = e10 < 0 ? '-' : '+';
        body[n++] = (char)('0' + ae / 10);
        body[n++] = (char)('0' + ae % 10);
    } else {
        body[n++] = e10 < 0 ? '-' : '+';
        body[n++] = (char)('0' + ae / 100);
        body[n++] = (char)('0' + (ae / 10) % 10);
        body[n++] = (char)('0' + ae % 10);
    }
    // right-justified in 15 columns; a longer body keeps its first 15 characters
    if (n >= 15) {
        std::memcpy(field, body, 15);
    } else {
        std::memset(field, ' ', (size_t)(15 - n));
        std::memcpy(field + 15 - n, body, (size_t)n);
    }
    field[15] = 0;
}

}  // namespace

extern "C" {

void ysh_format_e15_6(double x, char field[16]) { e15_6_fast(x, field); }

int ysh_event_setup(const ysh_model* m, const ysh_params* p, ysh_event* e)
{
    std::memset(e, 0, sizeof *e);
    ysh_norms nm;
    ysh_norms_get(&nm);
    const double rtop = m->r[m->nknot - 1];
    // normalise the inputs, yspec.f90:179-189
    double f1 = p->f1 * nm.t_norm / 1000.0, f2 = p->f2 * nm.t_norm / 1000.0;
    double dt = p->dt / nm.t_norm;
    double rs = rtop - p->depth_s * 1000.0 / nm.r_norm;
    double rr = rtop - p->depth_r * 1000.0 / nm.r_norm;
    double tout = p->tout * 60.0 / nm.t_norm;
    // fcal, module_fourier.f90:362-397 (float log and truncations kept)
    if (0.5 / dt < f2) return YSH_ERR_NYQUIST;
    double ep = 5.0 / tout;
    double df = ep / (kTwoPi * 1.0);
    int nt = (int)(1.0 / (df * dt));
    int ne = (int)(std::log((float)nt) / std::log(2.0f) + 1.0f);
    nt = 1 << ne;
    df = 1.0 / ((double)nt * dt);
    int i1 = std::max((int)std::floor(f1 / df), 2);
    int i2 = (int)std::floor(f2 / df) + 2;
    double dw = kTwoPi * df;                                     // yspec.f90:200-205
    if (i1 == i2) return YSH_ERR_FEW_FREQ;
    int nw = i2 - i1 + 1;
    if (nw == 1) return YSH_ERR_FEW_FREQ;
    int is = radius_index(m, rs), ir = radius_index(m, rr);      // :210-215
    if (is == 0) return YSH_ERR_SRC_MODEL;
    if (is > m->nsl) return YSH_ERR_SRC_OCEAN;
    if (ir == 0) return YSH_ERR_REC_MODEL;
    if (ir > m->nsl) return YSH_ERR_REC_OCEAN;
    // geometry, :144-150
    int nr = p->nr;
    e->delta = (double*)std::calloc((size_t)std::max(nr, 1), sizeof(double));
    e->azst = (double*)std::calloc((size_t)std::max(nr, 1), sizeof(double));
    e->azep = (double*)std::calloc((size_t)std::max(nr, 1), sizeof(double));
    double lats = p->lat_s == 90.0 ? 89.98 : p->lat_s;
    for (int i = 0; i < nr; i++) {
        delaz(p->lat_r[i], p->lon_r[i], lats, p->lon_s, &e->delta[i], &e->azep[i], &e->azst[i]);
        e->azep[i] = kTwoPi - e->azep[i];
        e->azst[i] = kPi - e->azst[i];
    }
    ysg_event& ev = e->ev;
    ev.lmin = p->lmin;
    ev.lmax = p->lmax;
    ev.nw = nw;
    ev.is = is;
    ev.ir = ir;
    ev.ats = p->ats;
    ev.grav = p->grav;
    ev.out = p->out;
    ev.cor = p->cor;
    ev.nr = nr;
    ev.jofs = 0;
    ev.jstride = 1;
    ev.wmin = (double)(i1 - 1) * dw;
    ev.dw = dw;
    ev.ep = ep;
    ev.rs = rs;
    ev.rr = rr;
    for (int i = 0; i < 6; i++) ev.mm[i] = p->mm[i] / nm.moment_norm;
    ev.delta = e->delta;
    ev.azst = e->azst;
    ysg_time& tm = e->tm;
    tm.nt = nt;
    tm.i1 = i1;
    tm.i2 = i2;
    tm.nr = nr;
    tm.df = df;
    tm.dt = dt;
    tm.ep = ep;
    tm.tout = tout;
    tm.f11 = p->f11 / 1000.0 * nm.t_norm;
    tm.f12 = p->f12 / 1000.0 * nm.t_norm;
    tm.f21 = p->f21 / 1000.0 * nm.t_norm;
    tm.f22 = p->f22 / 1000.0 * nm.t_norm;
    tm.t_norm = nm.t_norm;
    tm.amp_norm = p->out == 0 ? nm.r_norm : (p->out == 1 ? nm.vel_norm : nm.acl_norm);
    tm.azep = e->azep;
    e->nt = nt;
    e->i1 = i1;
    e->i2 = i2;
    return YSH_OK;
}

void ysh_free_event(ysh_event* e)
{
    std::free(e->delta);
    std::free(e->azst);
    std::free(e->azep);
    e->delta = e->azst = e->azep = nullptr;
}

// One receiver's file (yspec.f90:488-503): nout lines of ncol E15.6
// fields, the file name the prefix, a dot and the receiver number.
static bool write_one(const std::string& pref, const double* out, int nout, int ncol, int k)
{
    // string_cat_int: digits counted with a single-precision log10
    char num[16];
    std::snprintf(num, sizeof num, "%10d", k);
    int j = (int)std::floor(std::log10((float)k));
    std::string path = pref + "." + std::string(num + 9 - j);
    std::string text;
    text.reserve((size_t)nout * (15 * (size_t)ncol + 1));
    char f[16];
    const double* base = out + (size_t)nout * ncol * (size_t)(k - 1);
    for (int i = 0; i < nout; i++) {
        for (int c = 0; c < ncol; c++) {
            e15_6_fast(base[(size_t)i + (size_t)nout * c], f);
            text.append(f, 15);
        }
        text += '\n';
    }
    std::FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) return false;
    const bool ok = std::fwrite(text.data(), 1, text.size(), fp) == text.size();
    return std::fclose(fp) == 0 && ok;
}

// The files of nr receivers, (nout, ncol, nr) column-major, on threads.
static int write_files_of(const std::string& pref, const double* out, int nout, int ncol, int nr)
{
    // Receivers are independent files: format and write them on several
    // threads (the text conversion dominates at thousands of receivers).
    unsigned hw = std::thread::hardware_concurrency();
    int nth = (int)std::min<unsigned>(hw ? hw : 1, 32u);
    nth = std::max(1, std::min(nth, nr / 4));
    std::atomic<int> next{1};
    std::atomic<bool> ok{true};
    auto work = [&]() {
        for (int k = next++; k <= nr; k = next++)
            if (!write_one(pref, out, nout, ncol, k)) ok = false;
    };
    if (nth == 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; t++) pool.emplace_back(work);
        for (auto& t : pool) t.join();
    }
    return ok ? YSH_OK : YSH_ERR_IO;
}

int ysh_write_traces(const char* pref_out, const double* out, int nout, int nr)
{
    return write_files_of(pref_out, out, nout, 4, nr);
}

int ysh_write_potential(const char* pref_out, const double* out, int nout, int nr)
{
    return write_files_of(std::string(pref_out) + ".pot", out, nout, 2, nr);
}

// Wall-clock seconds, for the per-phase report of YSPEC_TIMING.
static double wall_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int ysh_run(const char* param_file, int device, int write_files, double** out, int* nout, int* nr)
{
    const bool timing = std::getenv("YSPEC_TIMING") != nullptr;
    const double t0 = wall_s();
    double t1 = t0, t2 = t0, t3 = t0;
    if (out) *out = nullptr;
    ysh_params p;
    int rc = ysh_read_params(param_file, &p);
    if (rc) return rc;
    ysh_model* m = nullptr;
    rc = ysh_read_model(p.model_file, &m);
    if (rc) {
        ysh_free_params(&p);
        return rc;
    }
    ysh_event e;
    rc = ysh_event_setup(m, &p, &e);
    ysg_handle* h = nullptr;
    double* buf = nullptr;
    int no = 0;
    if (!rc) rc = ysg_create(&h, device);
    // one run per handle: no autotuning (it would solve the event once per
    // schedule); schedule 2 is the autotuner's choice on every measured workload
    if (!rc) rc = ysg_set_schedule(h, 2);
    if (!rc) {
        ysg_model view;
        ysh_model_view(m, &view);
        rc = ysg_model_upload(h, &view);
    }
    if (!rc) {
        int rows = ysg_trace_rows(&e.tm);
        buf = (double*)std::malloc((size_t)rows * 4 * (size_t)std::max(p.nr, 1) * sizeof(double));
        t1 = wall_s();
        rc = ysg_event_run(h, &e.ev, &e.tm, buf, &no);
        t2 = wall_s();
    }
    if (!rc && write_files) rc = ysh_write_traces(p.pref_out, buf, no, p.nr);
    t3 = wall_s();
    if (timing && !rc) {
        float ms[4] = {0, 0, 0, 0};
        ysg_last_timings(h, ms);
        std::fprintf(stderr,
                     "yspec timing: setup %.3f s (parameters, model, geometry, device, upload), "
                     "engine %.3f s (device stages ms: Legendre %.2f, solves %.2f, l-sum %.2f, "
                     "time series %.2f), writer %.3f s (%d files x %d lines)\n",
                     t1 - t0, t2 - t1, ms[0], ms[1], ms[2], ms[3], t3 - t2, write_files ? p.nr : 0, no);
    }
    if (!rc && out) {
        *out = buf;
        buf = nullptr;
    }
    if (nout) *nout = no;
    if (nr) *nr = p.nr;
    std::free(buf);
    if (h) ysg_destroy(h);
    ysh_free_event(&e);
    ysh_free_model(m);
    ysh_free_params(&p);
    return rc;
}

int ysh_run_potential(const char* param_file, int device, int write_files, double** out, int* nout, int* nr)
{
    if (out) *out = nullptr;
    ysh_params p;
    int rc = ysh_read_params(param_file, &p);
    if (rc) return rc;
    ysh_model* m = nullptr;
    rc = ysh_read_model(p.model_file, &m);
    if (rc) {
        ysh_free_params(&p);
        return rc;
    }
    ysh_event e;
    rc = ysh_event_setup(m, &p, &e);
    ysg_handle* h = nullptr;
    double* buf = nullptr;
    int no = 0;
    if (!rc) rc = ysg_create(&h, device);
    if (!rc) rc = ysg_set_schedule(h, 2);
    if (!rc) {
        ysg_model view;
        ysh_model_view(m, &view);
        rc = ysg_model_upload(h, &view);
    }
    if (!rc) {
        // the potential's normalisation for the output type (module_model.f90:489)
        ysh_norms nm;
        ysh_norms_get(&nm);
        ysg_time tm = e.tm;
        tm.amp_norm = nm.pot_norm / std::pow(nm.t_norm, (double)p.out);
        int rows = ysg_trace_rows(&tm);
        buf = (double*)std::malloc((size_t)rows * 2 * (size_t)std::max(p.nr, 1) * sizeof(double));
        rc = ysg_event_potential(h, &e.ev, &tm, buf, &no);
    }
    if (!rc && write_files) rc = ysh_write_potential(p.pref_out, buf, no, p.nr);
    if (!rc && out) {
        *out = buf;
        buf = nullptr;
    }
    if (nout) *nout = no;
    if (nr) *nr = p.nr;
    std::free(buf);
    if (h) ysg_destroy(h);
    ysh_free_event(&e);
    ysh_free_model(m);
    ysh_free_params(&p);
    return rc;
}

int ysh_run_batch(int nfiles, const char* const* param_files, int device, int write_files,
                  int* failed)
{
    if (failed) *failed = -1;
    if (nfiles < 1 || !param_files) return YSG_ERR_ARG;
    // read every parameter file first (the reference stops at the first bad one)
    std::vector<ysh_params> ps((size_t)nfiles);
    int rc = 0, nread = 0;
    for (; nread < nfiles; nread++) {
        rc = ysh_read_params(param_files[nread], &ps[(size_t)nread]);
        if (rc) {
            if (failed) *failed = nread;
            break;
        }
    }
    // events sharing a model deck run as one batch on the device
    std::map<std::string, std::vector<int>> groups;
    for (int i = 0; i < nread && !rc; i++) groups[ps[(size_t)i].model_file].push_back(i);
    ysg_handle* h = nullptr;
    if (!rc) rc = ysg_create(&h, device);
    // one run per handle: no autotuning (it would solve the event once per
    // schedule); schedule 2 is the autotuner's choice on every measured workload
    if (!rc) rc = ysg_set_schedule(h, 2);
    for (auto it = groups.begin(); it != groups.end() && !rc; ++it) {
        const std::vector<int>& ids = it->second;
        ysh_model* m = nullptr;
        rc = ysh_read_model(it->first.c_str(), &m);
        if (rc) {
            if (failed) *failed = ids[0];
            break;
        }
        std::vector<ysh_event> es(ids.size());
        size_t nset = 0;
        for (; nset < ids.size(); nset++) {
            rc = ysh_event_setup(m, &ps[(size_t)ids[nset]], &es[nset]);
            if (rc) {
                if (failed) *failed = ids[nset];
                break;
            }
        }
        std::vector<ysg_event> evs;
        std::vector<ysg_time> tms;
        std::vector<std::vector<double>> bufs(ids.size());
        std::vector<double*> outs;
        std::vector<int> nouts(ids.size(), 0);
        if (!rc) {
            ysg_model view;
            ysh_model_view(m, &view);
            rc = ysg_model_upload(h, &view);
        }
        if (!rc) {
            for (size_t e = 0; e < ids.size(); e++) {
                evs.push_back(es[e].ev);
                tms.push_back(es[e].tm);
                bufs[e].resize((size_t)ysg_trace_rows(&es[e].tm) * 4 * (size_t)std::max(es[e].ev.nr, 1));
                outs.push_back(bufs[e].data());
            }
            rc = ysg_batch_run(h, (int)ids.size(), evs.data(), tms.data(), outs.data(), nouts.data());
        }
        for (size_t e = 0; e < ids.size() && !rc && write_files; e++) {
            const ysh_params& p = ps[(size_t)ids[e]];
            rc = ysh_write_traces(p.pref_out, bufs[e].data(), nouts[e], p.nr);
            if (rc && failed) *failed = ids[e];
        }
        for (size_t e = 0; e < nset; e++) ysh_free_event(&es[e]);
        ysh_free_model(m);
    }
    if (h) ysg_destroy(h);
    for (int i = 0; i < nread; i++) ysh_free_params(&ps[(size_t)i]);
    return rc;
}

void ysh_free(void* ptr) { std::free(ptr); }

const char* ysh_status_string(int status)
{
    switch (status) {
        case YSH_OK: return "ok";
        case YSH_ERR_PARAM_FILE: return "can't find parameter file";
        case YSH_ERR_PARAM_READ: return "problem reading parameter file";
        case YSH_ERR_MODEL_FILE: return " problem opening model file";
        case YSH_ERR_MODEL_READ: return "problem reading model file";
        case YSH_ERR_NYQUIST: return "Nyquist frequency below fmax";
        case YSH_ERR_FEW_FREQ: return "too few frequency steps";
        case YSH_ERR_SRC_MODEL: return " source not in model!";
        case YSH_ERR_SRC_OCEAN: return " source in the ocean!";
        case YSH_ERR_REC_MODEL: return " receiver not in model!";
        case YSH_ERR_REC_OCEAN: return " receiver in the ocean!";
        case YSH_ERR_IO: return "could not write output file";
        default: return ysg_status_string(status);
    }
}

}  // extern "C"
