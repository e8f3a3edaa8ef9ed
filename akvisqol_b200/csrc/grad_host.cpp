// Host half of d MOS / d degraded signal; see grad_host.h.
#include "grad_host.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace vqb {
namespace host {

namespace {

constexpr double kC1g = (0.01 * 1.0) * (0.01 * 1.0);
constexpr double kC3g = (0.03 * 1.0) * (0.03 * 1.0) / 2.0;
// NSIM 3x3 window (reference src/nsim.zig:111-115); symmetric, so the flip
// of the taps does not matter here: weight of the neighbour (dr, dc).
constexpr double kWin[3][3] = {{0.0113033910173052, 0.0838251475442633, 0.0113033910173052},
                               {0.0838251475442633, 0.619485845753726, 0.0838251475442633},
                               {0.0113033910173052, 0.0838251475442633, 0.0113033910173052}};

inline size_t clampi(long v, size_t n) { return v < 0 ? 0 : (size_t)v >= n ? n - 1 : (size_t)v; }

// conv2d3x3Replicate (reference src/nsim.zig:204-218) in plain sums (the
// forward values feeding the partial derivatives; their rounding order is
// immaterial to a gradient).
void conv3(const double *in, double *out, size_t nr, size_t nc) {
    for (size_t r = 0; r < nr; ++r)
        for (size_t c = 0; c < nc; ++c) {
            double s = 0.0;
            for (int dr = -1; dr <= 1; ++dr)
                for (int dc = -1; dc <= 1; ++dc)
                    s += kWin[dr + 1][dc + 1] * in[clampi((long)r + dr, nr) * nc + clampi((long)c + dc, nc)];
            out[r * nc + c] = s;
        }
}

// conv3's adjoint: g_in[neighbour] += w * g_out[cell] (times scale[neighbour]
// when given), for every cell and tap, replicate padding included.
void conv3_adjoint(const double *g_out, const double *scale, double *g_in, size_t nr, size_t nc) {
    for (size_t r = 0; r < nr; ++r)
        for (size_t c = 0; c < nc; ++c) {
            const double g = g_out[r * nc + c];
            if (g == 0.0) continue;
            for (int dr = -1; dr <= 1; ++dr)
                for (int dc = -1; dc <= 1; ++dc) {
                    const size_t k = clampi((long)r + dr, nr) * nc + clampi((long)c + dc, nc);
                    g_in[k] += kWin[dr + 1][dc + 1] * g * (scale ? scale[k] : 1.0);
                }
        }
}

}  // namespace

double scores_grad(const std::vector<Match> &matches, size_t nb, double frame_duration, const Svr *svr, bool speech,
                   bool unscaled_speech, const LatticeMapper *lattice, std::vector<MatchGrad> &out) {
    const size_t n = matches.size();
    out.assign(n, MatchGrad{std::vector<double>(nb, 0.0), std::vector<double>(nb, 0.0), std::vector<double>(nb, 0.0)});
    const Scores s = build_scores(matches, nb, frame_duration, svr, speech, unscaled_speech, {}, 0.0, lattice);
    if (n == 0 || s.vnsim < 0.15) return s.moslqo;
    std::vector<double> dfv(nb, 0.0), dfv10(nb, 0.0), dfstd(nb, 0.0), denergy(nb, 0.0);
    if (!speech) {
        // predictClamped (reference src/svr.zig:56-67): sum_i coeff_i exp(-gamma |x - sv_i|^2) - rho in [1, 5]
        const double raw = svr->predict(s.fvnsim.data());
        if (raw < 1.0 || raw > 5.0) return s.moslqo;
        for (size_t i = 0; i < svr->coeff.size(); ++i) {
            double dist = 0.0;
            for (size_t f = 0; f < svr->nf; ++f) {
                const double d = svr->sv[i * svr->nf + f] - s.fvnsim[f];
                dist += d * d;
            }
            const double w = svr->coeff[i] * std::exp(-svr->gamma * dist) * 2.0 * svr->gamma;
            for (size_t f = 0; f < svr->nf && f < nb; ++f) dfv[f] += w * (svr->sv[i * svr->nf + f] - s.fvnsim[f]);
        }
    } else if (lattice) {
        // central differences over each of the mapper's 4 x nb features
        std::vector<double> f[4] = {s.fvnsim, s.fvnsim10, s.fstdnsim, s.fvdegenergy};
        std::vector<double> *g[4] = {&dfv, &dfv10, &dfstd, &denergy};
        for (int k = 0; k < 4; ++k)
            for (size_t b = 0; b < nb; ++b) {
                const double x = f[k][b], h = 1e-3 * std::max(1.0, std::fabs(x));
                f[k][b] = x + h;
                const double up = lattice->predict(f[0].data(), f[1].data(), f[2].data(), f[3].data());
                f[k][b] = x - h;
                const double dn = lattice->predict(f[0].data(), f[1].data(), f[2].data(), f[3].data());
                f[k][b] = x;
                (*g[k])[b] = (up - dn) / (2.0 * h);
            }
    } else {
        // exponential fit over mean NSIM (reference src/visqol.zig:85-96)
        double acc = 0.0;
        for (double x : s.fvnsim) acc += x;
        const double mean = acc / (double)nb;
        const double e = std::exp(0.0154302525 * (mean - -361.063949));
        const double gain = unscaled_speech ? 1.0 : (double)1.245063f;
        const double raw = (-262.847869 + e) * gain;
        if (raw < 1.0 || raw > 5.0) return s.moslqo;
        for (size_t b = 0; b < nb; ++b) dfv[b] = gain * 0.0154302525 * e / (double)nb;
    }
    // buildResult's reverse (reference src/visqol.zig:595-709)
    const double nf = (double)n;
    for (size_t p = 0; p < n; ++p)
        for (size_t b = 0; b < nb; ++b) {
            out[p].dmeans[b] += dfv[b] / nf;
            out[p].denergy[b] += denergy[b] / nf;
        }
    // fvnsim10: the k lowest means per band (the forward's sorted order,
    // first occurrences on ties)
    const size_t k = std::max<size_t>(1, (size_t)std::trunc(nf * 0.10));
    std::vector<size_t> order(n);
    for (size_t b = 0; b < nb; ++b) {
        if (dfv10[b] == 0.0) continue;
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t x, size_t y) { return matches[x].means[b] < matches[y].means[b]; });
        for (size_t i = 0; i < k; ++i) out[order[i]].dmeans[b] += dfv10[b] / (double)k;
    }
    // fstdnsim: sqrt((sum_p (fc_p - 1) sd^2 + fc_p m^2 - fvnsim^2 total) / (total - 1))
    int64_t frames = 0;
    std::vector<double> fc(n);
    for (size_t p = 0; p < n; ++p) {
        const int64_t c = (int64_t)std::ceil((matches[p].ref_end - matches[p].ref_start) / frame_duration);
        fc[p] = (double)c;
        frames += c;
    }
    const double total = (double)frames;
    for (size_t b = 0; b < nb; ++b) {
        if (dfstd[b] == 0.0 || !(s.fstdnsim[b] > 0.0)) continue;
        const double dv = dfstd[b] / (2.0 * s.fstdnsim[b]) / (total - 1.0);
        for (size_t p = 0; p < n; ++p) {
            const Match &m = matches[p];
            out[p].dstddevs[b] += dv * 2.0 * (fc[p] - 1.0) * m.stddevs[b];
            out[p].dmeans[b] += dv * (2.0 * fc[p] * m.means[b] - 2.0 * s.fvnsim[b] * total / nf);
        }
    }
    return s.moslqo;
}

void patch_similarity_grad(const double *ref, const double *deg, size_t nb, size_t nc, const double *dmeans,
                           const double *dstddevs, const double *denergy, double *dref, double *ddeg) {
    const size_t n = nb * nc;
    std::vector<double> mr(n), md(n), rsq(n), dsq(n), rd(n), crs(n), cds(n), crd(n);
    for (size_t i = 0; i < n; ++i) {
        rsq[i] = ref[i] * ref[i];
        dsq[i] = deg[i] * deg[i];
        rd[i] = ref[i] * deg[i];
    }
    conv3(ref, mr.data(), nb, nc);
    conv3(deg, md.data(), nb, nc);
    conv3(rsq.data(), crs.data(), nb, nc);
    conv3(dsq.data(), cds.data(), nb, nc);
    conv3(rd.data(), crd.data(), nb, nc);
    // the cells' similarities, then d loss / d similarity per cell
    std::vector<double> sim(n);
    for (size_t i = 0; i < n; ++i) {
        const double rms = mr[i] * mr[i], dms = md[i] * md[i], mrd = mr[i] * md[i];
        const double I = (2.0 * mrd + kC1g) / (rms + dms + kC1g);
        const double prod = (crs[i] - rms) * (cds[i] - dms);
        const double den = prod < 0.0 ? kC3g : std::sqrt(prod) + kC3g;
        sim[i] = I * ((crd[i] - mrd + kC3g) / den);
    }
    std::vector<double> dsim(n, 0.0);
    for (size_t r = 0; r < nb; ++r) {
        double mean = 0.0;
        for (size_t c = 0; c < nc; ++c) mean += sim[r * nc + c];
        mean /= (double)nc;
        double ss = 0.0;
        for (size_t c = 0; c < nc; ++c) ss += (sim[r * nc + c] - mean) * (sim[r * nc + c] - mean);
        const double sd = nc > 1 ? std::sqrt(ss / ((double)nc - 1.0)) : 0.0;
        for (size_t c = 0; c < nc; ++c) {
            double g = (dmeans ? dmeans[r] : 0.0) / (double)nc;
            if (dstddevs && sd > 0.0) g += dstddevs[r] * (sim[r * nc + c] - mean) / (((double)nc - 1.0) * sd);
            dsim[r * nc + c] = g;
            if (denergy) ddeg[r * nc + c] += denergy[r] / (double)nc;  // energy: the mean of the deg row
        }
    }
    // simCell's partials (reference src/nsim.zig:293-308), then the
    // windowed sums' adjoints
    std::vector<double> gmr(n, 0.0), gmd(n, 0.0), gcrs(n, 0.0), gcds(n, 0.0), gcrd(n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        if (dsim[i] == 0.0) continue;
        const double rms = mr[i] * mr[i], dms = md[i] * md[i], mrd = mr[i] * md[i];
        const double nn = 2.0 * mrd + kC1g, dd = rms + dms + kC1g;
        const double I = nn / dd;
        const double srs = crs[i] - rms, sds = cds[i] - dms, srd = crd[i] - mrd;
        const double prod = srs * sds;
        const double den = prod < 0.0 ? kC3g : std::sqrt(prod) + kC3g;
        const double S = (srd + kC3g) / den;
        const double dI = dsim[i] * S, dS = dsim[i] * I;
        const double dI_mr = (2.0 * md[i] * dd - nn * 2.0 * mr[i]) / (dd * dd);
        const double dI_md = (2.0 * mr[i] * dd - nn * 2.0 * md[i]) / (dd * dd);
        double dS_srs = 0.0, dS_sds = 0.0;
        if (prod > 0.0) {
            const double q = -(srd + kC3g) / (den * den) / (2.0 * std::sqrt(prod));
            dS_srs = q * sds;
            dS_sds = q * srs;
        }
        gmr[i] = dI * dI_mr + dS * (-md[i] / den) + dS * dS_srs * (-2.0 * mr[i]);
        gmd[i] = dI * dI_md + dS * (-mr[i] / den) + dS * dS_sds * (-2.0 * md[i]);
        gcrd[i] = dS / den;
        gcrs[i] = dS * dS_srs;
        gcds[i] = dS * dS_sds;
    }
    // mu_ref <- ref, mu_deg <- deg, conv(ref^2), conv(deg^2), conv(ref*deg)
    std::vector<double> two_ref(n), two_deg(n);
    for (size_t i = 0; i < n; ++i) two_ref[i] = 2.0 * ref[i], two_deg[i] = 2.0 * deg[i];
    conv3_adjoint(gmr.data(), nullptr, dref, nb, nc);
    conv3_adjoint(gmd.data(), nullptr, ddeg, nb, nc);
    conv3_adjoint(gcrs.data(), two_ref.data(), dref, nb, nc);
    conv3_adjoint(gcds.data(), two_deg.data(), ddeg, nb, nc);
    conv3_adjoint(gcrd.data(), deg, dref, nb, nc);
    conv3_adjoint(gcrd.data(), ref, ddeg, nb, nc);
}

namespace {
constexpr double kAbsFloor = -45.0, kRelFloor = 45.0;

double to_db(double x) {
    const double v = x == 0.0 ? std::numeric_limits<double>::epsilon() : std::fabs(x);
    return std::fmax(10.0 * std::log10(v), kAbsFloor);
}
}  // namespace

void prepare_forward(const double *ref_raw, const double *deg_raw, size_t nb, size_t nfr, size_t nfd,
                     std::vector<double> &ref, std::vector<double> &deg) {
    ref.resize(nb * nfr);
    deg.resize(nb * nfd);
    for (size_t i = 0; i < nb * nfr; ++i) ref[i] = to_db(ref_raw[i]);
    for (size_t i = 0; i < nb * nfd; ++i) deg[i] = to_db(deg_raw[i]);
    const size_t m = std::min(nfr, nfd);
    for (size_t c = 0; c < m; ++c) {
        double col = -std::numeric_limits<double>::infinity();
        for (size_t r = 0; r < nb; ++r) col = std::max(col, std::fmax(ref[r * nfr + c], deg[r * nfd + c]));
        const double floor = col - kRelFloor;
        for (size_t r = 0; r < nb; ++r) {
            ref[r * nfr + c] = std::max(ref[r * nfr + c], floor);
            deg[r * nfd + c] = std::max(deg[r * nfd + c], floor);
        }
    }
    double lo = std::numeric_limits<double>::infinity();
    for (double v : ref) lo = std::min(lo, v);
    for (double v : deg) lo = std::min(lo, v);
    for (double &v : ref) v -= lo;
    for (double &v : deg) v -= lo;
}

void prepare_grad(const double *ref_raw, const double *deg_raw, size_t nb, size_t nfr, size_t nfd,
                  const double *g_ref, const double *g_deg, double *g_deg_raw) {
    // forward replay with the selections: dB values, per-column floors and
    // their source cells, the joint minimum's cell
    std::vector<double> rdb(nb * nfr), ddb(nb * nfd), rv, dv;
    for (size_t i = 0; i < nb * nfr; ++i) rdb[i] = to_db(ref_raw[i]);
    for (size_t i = 0; i < nb * nfd; ++i) ddb[i] = to_db(deg_raw[i]);
    rv = rdb;
    dv = ddb;
    const size_t m = std::min(nfr, nfd);
    std::vector<double> floor(m);
    std::vector<long> src(m, -1);  // deg cell that set the column's floor, or -1 (a ref cell)
    for (size_t c = 0; c < m; ++c) {
        double col = -std::numeric_limits<double>::infinity();
        long s = -1;
        for (size_t r = 0; r < nb; ++r) {
            const double a = rdb[r * nfr + c], b = ddb[r * nfd + c];
            const double v = std::fmax(a, b);
            if (v > col) {
                col = v;
                s = b > a ? (long)(r * nfd + c) : -1;
            }
        }
        floor[c] = col - kRelFloor;
        src[c] = s;
        for (size_t r = 0; r < nb; ++r) {
            rv[r * nfr + c] = std::max(rv[r * nfr + c], floor[c]);
            dv[r * nfd + c] = std::max(dv[r * nfd + c], floor[c]);
        }
    }
    // joint minimum: first minimum, ref cells before deg cells
    double lo = std::numeric_limits<double>::infinity();
    long lo_ref = -1, lo_deg = -1;
    for (size_t i = 0; i < nb * nfr; ++i)
        if (rv[i] < lo) lo = rv[i], lo_ref = (long)i, lo_deg = -1;
    for (size_t i = 0; i < nb * nfd; ++i)
        if (dv[i] < lo) lo = dv[i], lo_deg = (long)i, lo_ref = -1;
    double total = 0.0;
    for (size_t i = 0; i < nb * nfr; ++i) total += g_ref[i];
    for (size_t i = 0; i < nb * nfd; ++i) total += g_deg[i];
    // gradients of the floored values (before the minimum's subtraction)
    std::vector<double> gr(g_ref, g_ref + nb * nfr), gd(g_deg, g_deg + nb * nfd);
    if (lo_ref >= 0) gr[lo_ref] -= total;
    if (lo_deg >= 0) gd[lo_deg] -= total;
    // floors: a floored cell's gradient goes to the cell that set the floor
    std::vector<double> gddb(nb * nfd, 0.0);
    for (size_t i = 0; i < nb * nfd; ++i) {
        const size_t c = i % nfd;
        if (c < m && ddb[i] < floor[c]) {
            if (src[c] >= 0) gddb[src[c]] += gd[i];
        } else {
            gddb[i] += gd[i];
        }
    }
    for (size_t i = 0; i < nb * nfr; ++i) {
        const size_t c = i % nfr;
        if (c < m && rdb[i] < floor[c] && src[c] >= 0) gddb[src[c]] += gr[i];
    }
    // dB: 10 log10|x| above the absolute floor
    for (size_t i = 0; i < nb * nfd; ++i) {
        const double x = deg_raw[i];
        if (gddb[i] == 0.0 || x == 0.0) continue;
        if (10.0 * std::log10(std::fabs(x)) < kAbsFloor) continue;
        g_deg_raw[i] += gddb[i] * 10.0 / (x * std::log(10.0));
    }
}

}  // namespace host
}  // namespace vqb
