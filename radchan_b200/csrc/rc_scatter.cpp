// rc_scatter.cpp -- particle scattering tables on the host: the seeded
// synthetic builder, the reader and writer of the table generator's particle
// files, and the checks the march relies on.
//
// Formats (nbcorrk/write_tables.cpp):
//   NarrBand%d.txt   writeP (:204-260): "wvl wvr wvc", then the nQ particle
//                    absorption coefficients, then the nQ scattering ones;
//   prob_scatt.txt   writeH (:326-336): "theta wvc cdf" for every band and
//                    angle, angles fastest.
// The phase-function CDF follows calc_prob.cpp:253-270: trapezoids of
// p(theta) sin(theta) between table angles, accumulated and normalised by the
// last entry.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <cctype>
#include <string>
#include <vector>

#include "radchan_math.h"
#include "rc_host.h"

namespace rc {

void ScatterSet::view(rc_scattering *s) const {
    s->nB = nB;
    s->nQ = nQ;
    s->nA = nA;
    s->ksca = ksca.data();
    s->kabs = kabs.empty() ? nullptr : kabs.data();
    s->theta = theta.data();
    s->phase_cdf = cdf.data();
}

namespace {

// CDF over the angles of one band from its phase function samples p[nA]
// (calc_prob.cpp:253-270).
void phase_cdf_from_samples(const std::vector<double> &th, const std::vector<double> &p, float *cdf) {
    const int nA = (int)th.size();
    std::vector<double> c(nA, 0.0);
    for (int t = 1; t < nA; ++t) {
        const double pr = 0.5 * (th[t] - th[t - 1]) * (p[t] + p[t - 1]) * 0.5 * (sin(th[t]) + sin(th[t - 1])) * 0.5;
        c[t] = c[t - 1] + pr;
    }
    const double last = c[nA - 1];
    for (int t = 0; t < nA; ++t) cdf[t] = (float)(c[t] / last);
    cdf[nA - 1] = 1.0f;
}

bool read_all_numbers(const std::string &path, std::vector<double> &v) {
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return false;
    v.clear();
    std::string tok;
    int ch;
    while ((ch = fgetc(f)) != EOF) {
        if (isspace(ch)) {
            if (!tok.empty()) {
                v.push_back(strtod(tok.c_str(), nullptr));
                tok.clear();
            }
        } else {
            tok += (char)ch;
        }
    }
    if (!tok.empty()) v.push_back(strtod(tok.c_str(), nullptr));
    fclose(f);
    return true;
}

}  // namespace

int scattering_synthetic(const rc_scatter_spec &s, ScatterSet &out, std::string &err) {
    if (s.nB < 1 || s.nQ < 1 || s.nA < 2 || s.nA > 4096) {
        err = "invalid particle table dimensions";
        return RC_E_INVALID;
    }
    if (!(s.ksca_lo >= 0.0) || !(s.ksca_hi >= s.ksca_lo) || !(s.g_lo > -1.0) || !(s.g_hi < 1.0) ||
        !(s.g_hi >= s.g_lo)) {
        err = "invalid particle table recipe (0 <= ksca_lo <= ksca_hi, -1 < g_lo <= g_hi < 1)";
        return RC_E_INVALID;
    }
    out = ScatterSet();
    out.nB = s.nB;
    out.nQ = s.nQ;
    out.nA = s.nA;
    out.wvl.assign(s.nB, 0.f);
    out.wvr.assign(s.nB, 0.f);
    out.wvc.assign(s.nB, 0.f);
    out.kabs.assign((size_t)s.nB * s.nQ, 0.f);
    out.ksca.resize((size_t)s.nB * s.nQ);
    out.theta.resize(s.nA);
    out.cdf.resize((size_t)s.nB * s.nA);
    std::vector<double> th(s.nA), p(s.nA);
    for (int a = 0; a < s.nA; ++a) {
        th[a] = RC_PI_D * a / (s.nA - 1);
        out.theta[a] = (float)th[a];
    }
    for (int b = 0; b < s.nB; ++b) {
        double k;
        if (s.ksca_lo > 0.0 && s.ksca_hi > s.ksca_lo)
            k = exp(log(s.ksca_lo) + (log(s.ksca_hi) - log(s.ksca_lo)) * synth_uniform(s.seed, 11, b));
        else
            k = s.ksca_lo + (s.ksca_hi - s.ksca_lo) * synth_uniform(s.seed, 11, b);
        for (int g = 0; g < s.nQ; ++g) out.ksca[(size_t)b * s.nQ + g] = (float)k;
        const double gb = s.g_lo + (s.g_hi - s.g_lo) * synth_uniform(s.seed, 12, b);
        for (int a = 0; a < s.nA; ++a) p[a] = (1.0 - gb * gb) / pow(1.0 + gb * gb - 2.0 * gb * cos(th[a]), 1.5);
        phase_cdf_from_samples(th, p, &out.cdf[(size_t)b * s.nA]);
    }
    return RC_OK;
}

int scattering_read_dir(const std::string &dir, int nB, int nQ, ScatterSet &out, std::string &err) {
    if (nB < 1 || nQ < 1) {
        err = "invalid particle table dimensions";
        return RC_E_INVALID;
    }
    out = ScatterSet();
    out.nB = nB;
    out.nQ = nQ;
    out.wvl.resize(nB);
    out.wvr.resize(nB);
    out.wvc.resize(nB);
    out.kabs.resize((size_t)nB * nQ);
    out.ksca.resize((size_t)nB * nQ);
    std::vector<double> v;
    for (int b = 0; b < nB; ++b) {
        const std::string f = dir + "/NarrBand" + std::to_string(b) + ".txt";
        if (!read_all_numbers(f, v) || v.size() < (size_t)3 + 2 * (size_t)nQ) {
            err = "missing or short " + f;
            return RC_E_IO;
        }
        out.wvl[b] = (float)v[0];
        out.wvr[b] = (float)v[1];
        out.wvc[b] = (float)v[2];
        for (int g = 0; g < nQ; ++g) {
            out.kabs[(size_t)b * nQ + g] = (float)v[3 + g];
            out.ksca[(size_t)b * nQ + g] = (float)v[3 + nQ + g];
        }
    }
    const std::string f = dir + "/prob_scatt.txt";
    if (!read_all_numbers(f, v) || v.size() % 3 != 0 || v.size() / 3 < (size_t)2 * nB || (v.size() / 3) % nB != 0) {
        err = "missing or malformed " + f + " (3 numbers per row, a whole number of angles per band)";
        return RC_E_IO;
    }
    const int nA = (int)(v.size() / 3 / nB);
    if (nA > 4096) {
        err = "more than 4096 angles in " + f;
        return RC_E_IO;
    }
    out.nA = nA;
    out.theta.resize(nA);
    out.cdf.resize((size_t)nB * nA);
    for (int a = 0; a < nA; ++a) out.theta[a] = (float)v[3 * (size_t)a];
    for (int b = 0; b < nB; ++b)
        for (int a = 0; a < nA; ++a) {
            const double *r = &v[3 * ((size_t)b * nA + a)];
            if ((float)r[0] != out.theta[a]) {
                err = f + ": band " + std::to_string(b) + " lists other angles than band 0";
                return RC_E_IO;
            }
            out.cdf[(size_t)b * nA + a] = (float)r[2];
        }
    return RC_OK;
}

int scattering_write_dir(const ScatterSet &s, const std::string &dir, std::string &err) {
    for (int b = 0; b < s.nB; ++b) {
        const std::string f = dir + "/NarrBand" + std::to_string(b) + ".txt";
        FILE *fp = fopen(f.c_str(), "wt");
        if (!fp) {
            err = "cannot write " + f;
            return RC_E_IO;
        }
        fprintf(fp, "%le\t%le\t%le \n", (double)s.wvl[b], (double)s.wvr[b], (double)s.wvc[b]);
        for (int g = 0; g < s.nQ; ++g) fprintf(fp, " %le\t", s.kabs.empty() ? 0.0 : (double)s.kabs[(size_t)b * s.nQ + g]);
        fprintf(fp, "\n");
        for (int g = 0; g < s.nQ; ++g) fprintf(fp, " %le\t", (double)s.ksca[(size_t)b * s.nQ + g]);
        fclose(fp);
    }
    const std::string f = dir + "/prob_scatt.txt";
    FILE *fp = fopen(f.c_str(), "w+");
    if (!fp) {
        err = "cannot write " + f;
        return RC_E_IO;
    }
    // nine significant digits: a float written and read back is the same float
    for (int b = 0; b < s.nB; ++b)
        for (int a = 0; a < s.nA; ++a)
            fprintf(fp, "%.9e\t%le\t%.9e\n", (double)s.theta[a], (double)s.wvc[b], (double)s.cdf[(size_t)b * s.nA + a]);
    fclose(fp);
    return RC_OK;
}

int scattering_check(const rc_scattering &s, std::string &err) {
    char m[200];
    if (s.nB < 1 || s.nQ < 1 || s.nA < 2 || s.nA > 4096) {
        snprintf(m, sizeof(m), "particle table dimensions nB=%d nQ=%d nA=%d (need nB, nQ >= 1, 2 <= nA <= 4096)", s.nB,
                 s.nQ, s.nA);
        err = m;
        return RC_E_INVALID;
    }
    if (!s.ksca || !s.theta || !s.phase_cdf) {
        err = "NULL particle table array";
        return RC_E_INVALID;
    }
    for (int i = 0; i < s.nB * s.nQ; ++i)
        if (!(s.ksca[i] >= 0.0f) || !std::isfinite(s.ksca[i])) {
            snprintf(m, sizeof(m), "scattering coefficient %d (band %d, g %d) is %g: must be finite and >= 0", i,
                     i / s.nQ, i % s.nQ, (double)s.ksca[i]);
            err = m;
            return RC_E_INVALID;
        }
    for (int a = 0; a < s.nA; ++a) {
        const float t = s.theta[a];
        const bool ok = std::isfinite(t) && (a == 0 ? t >= 0.0f : t > s.theta[a - 1]) &&
                        (double)t <= RC_PI_D + 1e-6;
        if (!ok) {
            snprintf(m, sizeof(m), "scattering angle %d is %g: angles must increase from >= 0 to <= pi", a, (double)t);
            err = m;
            return RC_E_INVALID;
        }
    }
    for (int b = 0; b < s.nB; ++b) {
        const float *c = s.phase_cdf + (size_t)b * s.nA;
        for (int a = 0; a < s.nA; ++a) {
            const bool ok = std::isfinite(c[a]) && (a == 0 ? c[a] == 0.0f : c[a] >= c[a - 1]);
            if (!ok) {
                snprintf(m, sizeof(m), "phase CDF of band %d at angle %d is %g: must be 0 at the first angle, "
                                       "finite and non-decreasing", b, a, (double)c[a]);
                err = m;
                return RC_E_INVALID;
            }
        }
        if (!(fabs((double)c[s.nA - 1] - 1.0) <= 1e-6)) {
            snprintf(m, sizeof(m), "phase CDF of band %d ends at %.9g, not 1", b, (double)c[s.nA - 1]);
            err = m;
            return RC_E_INVALID;
        }
    }
    return RC_OK;
}

}  // namespace rc
