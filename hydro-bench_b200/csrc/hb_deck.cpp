// hb_deck.cpp -- reader for hydro-cal text decks, producing the arrays the
// reference uploads to the device.
//
// Follows cuda_native_impl/hydro-cal-src/src/mesh.cpp:
//   InitFromFile            :5-38     scalar files and the per-cell/per-slot files
//   loadFromFile*           :40-278   one record per line, header line first
//   preCalculate            :280-372  areas, side lengths, normals, initial depth
//   take_boundary_for_two_d :374-521  level/discharge series per table interval,
//                                     rating curves
//   BOUNDRYinterp           :523-533
// and the device relayout of cell.cpp:72-128 (per-day tables [NDAYS][CELL],
// rating tables [CELL][NHQ], BoundaryFeature from MBW).
//
// Numbers are parsed with strtod/strtol, which round exactly like the
// reference's istringstream extraction.  Host arithmetic is plain IEEE double
// (this file is compiled without FMA contraction), as in the reference.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "hydrob200.h"

namespace hb {
int set_error(int status, const char *fmt, ...);
}

struct hb_deck {
    int cells = 0, nod = 0, ndays = 0, mdt = 0, ntoutput = 0;
    int nz = 0, nq = 0, nzq = 0, nhq = 0, nwe = 0, ndi = 0;
    double dt = 0, hm1 = 0, hm2 = 0, jl = 0;
    std::vector<double> nac, klas, side, cosf, sinf, slcos, slsin;            // [4C]
    std::vector<double> h, u, v, z, w, zbc, zb1, area, fnc, bfeat;            // [C]
    std::vector<int32_t> nhq1;                                                // [C]
    std::vector<double> zw, qw;                                               // [C*NHQ]
    std::vector<double> qt, dqt, zt, dzt;                                     // [NDAYS*C]
    // for the OUTPUT writers
    std::vector<double> xp, yp;                                               // [NOD] node coordinates - (XIMIN, YIMIN)
    double ximin = 0, yimin = 0;
    std::vector<int32_t> nap;                                                 // [4C] node ids as read
};

namespace {

struct LineFile {
    std::vector<std::string> lines;
    size_t next = 0;
    bool ok = false;
    LineFile(const std::string &path) {
        std::ifstream f(path, std::ios::binary);
        if (!f.is_open()) return;
        std::string ln;
        while (std::getline(f, ln)) {
            if (!ln.empty() && ln.back() == '\r') ln.pop_back();
            lines.push_back(ln);
        }
        ok = true;
    }
    const char *get() { return next < lines.size() ? lines[next++].c_str() : nullptr; }
};

bool num_d(const char *&p, double &out) {
    char *e;
    double v = strtod(p, &e);
    if (e == p) return false;
    out = v; p = e; return true;
}
bool num_i(const char *&p, int &out) {
    char *e;
    long v = strtol(p, &e, 10);
    if (e == p) return false;
    out = (int)v; p = e; return true;
}

struct Series { std::vector<double> t, v; };

// mesh.cpp:523-533; the scan stops where the table ends (the reference reads
// one element past it when t reaches the last time)
double interp(double t, const Series &s) {
    double r = 0;
    const size_t n = s.t.size();
    for (size_t i = 1; i < n; i++)
        if (t >= s.t[i - 1] && t <= s.t[i]) r = s.v[i - 1] + (s.v[i] - s.v[i - 1]) / (s.t[i] - s.t[i - 1]) * (t - s.t[i - 1]);
    return r;
}

bool read_series(const std::string &path, Series &s, size_t min_cap) {
    LineFile f(path);
    if (!f.ok) return false;
    int n = 0;
    const char *ln = f.get();
    if (!ln || !num_i(ln, n) || n < 0) return false;
    s.t.assign(std::max<size_t>((size_t)n, min_cap), 0.0);
    s.v.assign(std::max<size_t>((size_t)n, min_cap), 0.0);
    for (int i = 0; i < n; i++) {
        ln = f.get();
        if (!ln) break;
        num_d(ln, s.t[i]);
        num_d(ln, s.v[i]);
    }
    s.t.resize(n); s.v.resize(n);
    return true;
}

int fail_io(const std::string &what) { return hb::set_error(HB_E_IO, "deck: cannot read %s", what.c_str()); }

}  // namespace

extern "C" int hb_deck_load(const char *root_c, hb_deck **out) {
    if (!root_c || !out) return hb::set_error(HB_E_INVALID, "hb_deck_load: null argument");
    const std::string root = std::string(root_c) + "/";
    auto d = new hb_deck();
    auto scal_i = [&](const char *rel, std::initializer_list<int *> dst) -> bool {
        LineFile f(root + rel);
        if (!f.ok) return false;
        for (int *p : dst) { const char *ln = f.get(); if (!ln || !num_i(ln, *p)) return false; }
        return true;
    };
    int dummy = 0;
    bool ok = scal_i("BINFOR/TIME.DAT", {&d->mdt, &d->ndays, &d->ntoutput}) &&
              scal_i("BINFOR/GIRD.DAT", {&d->nod, &d->cells}) &&
              scal_i("BINFOR/BOUNDARY.DAT", {&d->nz, &d->nq, &d->nzq, &d->nhq, &d->nwe, &d->ndi});
    if (ok) {
        LineFile f(root + "BINFOR/DEPTH.DAT");
        const char *a = f.ok ? f.get() : nullptr; const char *b = f.ok ? f.get() : nullptr;
        ok = a && b && num_d(a, d->hm1) && num_d(b, d->hm2);
    }
    if (ok) {
        LineFile f(root + "BINFOR/CALTIME.DAT");
        const char *a = f.ok ? f.get() : nullptr; const char *b = f.ok ? f.get() : nullptr;
        ok = a && b && num_i(a, dummy) && num_d(b, d->dt);
    }
    if (ok) {
        LineFile f(root + "BINFOR/JL.DAT");
        const char *a = f.ok ? f.get() : nullptr;
        ok = a && num_d(a, d->jl);
    }
    if (!ok) { delete d; return fail_io(root + "BINFOR/*.DAT"); }
    const int C = d->cells;
    if (C <= 0 || d->nod <= 0 || d->ndays <= 0 || d->nz < 0 || d->nq < 0 || d->nzq < 0 || d->nhq < 0 || d->dt <= 0) {
        delete d;
        return hb::set_error(HB_E_BADMESH, "deck: bad sizes (CELL=%d NOD=%d NDAYS=%d)", C, d->nod, d->ndays);
    }
    const size_t S = 4 * (size_t)C;
    d->nac.assign(S, 0); d->klas.assign(S, 0);
    std::vector<int> nap(S, 0);
    auto cell4 = [&](const char *rel, double *dst_d, int *dst_i) -> bool {
        LineFile f(root + rel);
        if (!f.ok) return false;
        f.get();
        for (int i = 0; i < C; i++) {
            const char *ln = f.get();
            if (!ln) break;
            int no;
            if (!num_i(ln, no)) continue;
            for (int j = 0; j < 4; j++) {
                if (dst_d) { if (!num_d(ln, dst_d[4 * i + j])) break; }
                else if (!num_i(ln, dst_i[4 * i + j])) break;
            }
        }
        return true;
    };
    auto column = [&](const char *rel, std::vector<double> &dst, int n) -> bool {
        LineFile f(root + rel);
        if (!f.ok) return false;
        dst.assign(n, 0.0);
        f.get();
        for (int i = 0; i < n; i++) {
            const char *ln = f.get();
            if (!ln) break;
            num_d(ln, dst[i]);
        }
        return true;
    };
    auto groups = [&](const char *rel, int rows, int &count0, std::vector<double> &c1, std::vector<double> &c2) -> bool {
        LineFile f(root + rel);
        if (!f.ok) return false;
        c1.assign(rows, 0.0); c2.assign(rows, 0.0);
        const char *ln = f.get();
        if (ln) num_i(ln, count0);
        for (int i = 0; i < rows; i++) {
            ln = f.get();
            if (!ln) break;
            int no;
            if (!num_i(ln, no)) continue;
            num_d(ln, c1[i]);
            num_d(ln, c2[i]);
        }
        return true;
    };
    std::vector<double> xp(d->nod, 0.0), yp(d->nod, 0.0), fnc0;
    std::vector<double> mbz, nnz, mbq, nnq, mbzq, nnzq, mbw, topw;
    int nnz0 = 0, nnq0 = 0, nnzq0 = 0;
    ok = cell4("SOURCES/PNAC.DAT", d->nac.data(), nullptr) && cell4("SOURCES/PNAP.DAT", nullptr, nap.data()) &&
         cell4("SOURCES/PKLAS.DAT", d->klas.data(), nullptr) && column("SOURCES/PZBC.DAT", d->zbc, C);
    if (ok) {
        LineFile f(root + "SOURCES/PXY.DAT");
        ok = f.ok;
        if (ok) {
            f.get();
            for (int i = 0; i < d->nod; i++) {
                const char *ln = f.get();
                if (!ln) break;
                int no;
                if (!num_i(ln, no)) continue;
                num_d(ln, xp[i]);
                num_d(ln, yp[i]);
            }
        }
    }
    ok = ok && groups("SOURCES/MBZ.DAT", d->nz, nnz0, mbz, nnz) && groups("SOURCES/MBQ.DAT", d->nq, nnq0, mbq, nnq);
    if (ok) {   // MBW.DAT's first line overrides NWE (mesh.cpp:178-197)
        LineFile f(root + "SOURCES/MBW.DAT");
        ok = f.ok;
        if (ok) {
            const char *ln = f.get();
            if (ln) num_i(ln, d->nwe);
            if (d->nwe < 0) d->nwe = 0;
            mbw.assign(d->nwe, 0.0); topw.assign(d->nwe, 0.0);
            for (int i = 0; i < d->nwe; i++) {
                ln = f.get();
                if (!ln) break;
                int no;
                if (!num_i(ln, no)) continue;
                num_d(ln, mbw[i]);
                num_d(ln, topw[i]);
            }
        }
    }
    ok = ok && groups("SOURCES/MBZQ.DAT", d->nzq, nnzq0, mbzq, nnzq) &&
         column("BINFOR/INITIALLEVEL.DAT", d->z, C) && column("BINFOR/INITIALU1.DAT", d->u, C) &&
         column("BINFOR/INITIALV1.DAT", d->v, C) && column("BINFOR/CV.DAT", fnc0, C);
    if (!ok) { delete d; return fail_io(root + "SOURCES/*.DAT or BINFOR/INITIAL*.DAT"); }

    // ---- geometry (mesh.cpp:280-372) ----
    double ximin = xp[0], yimin = yp[0];
    for (int i = 1; i < d->nod; i++) { ximin = std::min(ximin, xp[i]); yimin = std::min(yimin, yp[i]); }
    for (int i = 0; i < d->nod; i++) { xp[i] -= ximin; yp[i] -= yimin; }
    d->ximin = ximin;
    d->yimin = yimin;
    d->zb1.assign(C, 0.0); d->area.assign(C, 0.0);
    d->side.assign(S, 0.0); d->sinf.assign(S, 0.0); d->cosf.assign(S, 0.0);
    d->slcos.assign(S, 0.0); d->slsin.assign(S, 0.0);
    std::vector<int> nv(C, 0);
    for (int i = 0; i < C; i++) {
        const int *np = &nap[4 * i];
        if (np[0] == 0) continue;
        d->zb1[i] = d->zbc[i] + d->hm1;
        nv[i] = (np[3] == 0 || np[3] == np[0]) ? 3 : 4;
        for (int j = 0; j < nv[i]; j++)
            if (np[j] < 1 || np[j] > d->nod) {
                delete d;
                return hb::set_error(HB_E_BADMESH, "deck: cell %d node %d out of range", i + 1, np[j]);
            }
        const double x1 = xp[np[0] - 1], x2 = xp[np[1] - 1], x3 = xp[np[2] - 1];
        const double y1 = yp[np[0] - 1], y2 = yp[np[1] - 1], y3 = yp[np[2] - 1];
        d->area[i] = std::fabs(((y3 - y1) * (x2 - x1) - (x3 - x1) * (y2 - y1)) / 2.0);
        if (nv[i] == 4) {
            const double x4 = xp[np[3] - 1], y4 = yp[np[3] - 1];
            d->area[i] += std::fabs(((y4 - y1) * (x3 - x1) - (x4 - x1) * (y3 - y1)) / 2.0);
        }
        for (int j = 0; j < nv[i]; j++) {
            const int n1 = np[j] - 1, n2 = np[(j + 1) % nv[i]] - 1;
            const double dx = xp[n1] - xp[n2];
            const double dy = yp[n2] - yp[n1];
            const size_t s = 4 * (size_t)i + j;
            d->side[s] = std::sqrt(dx * dx + dy * dy);
            if (d->side[s] > 0.0) {
                d->sinf[s] = dx / d->side[s];
                d->cosf[s] = dy / d->side[s];
            }
        }
    }
    for (int i = 0; i < C; i++) d->zb1[i] = d->zbc[i] + d->hm1;
    d->h.assign(C, 0.0); d->w.assign(C, 0.0); d->fnc.assign(C, 0.0);
    for (int i = 0; i < C; i++) {
        if (nap[4 * i] == 0) continue;
        if (d->z[i] <= d->zbc[i]) { d->h[i] = d->hm1; d->z[i] = d->zb1[i]; }
        else d->h[i] = d->z[i] - d->zbc[i];
    }
    for (int i = 0; i < C; i++) {
        d->fnc[i] = 9.81 * fnc0[i] * fnc0[i];
        for (int j = 0; j < nv[i]; j++) {
            const size_t s = 4 * (size_t)i + j;
            d->slcos[s] = d->side[s] * d->cosf[s];
            d->slsin[s] = d->side[s] * d->sinf[s];
        }
    }

    // ---- boundary tables (mesh.cpp:374-521), relaid as cell.cpp:93-128 ----
    const int ND = d->ndays, NZ = d->nz, NQ = d->nq, NZQ = d->nzq, NHQ = d->nhq;
    std::vector<double> ZT((size_t)NZ * ND, 0.0), QT((size_t)NQ * ND, 0.0);
    char rel[64];
    for (int k = 1; k <= nnz0; k++) {
        snprintf(rel, sizeof rel, "BOUNDE/NZ/NZ%04d.DAT", k);
        Series s;
        if (!read_series(root + rel, s, 0)) { delete d; return fail_io(root + rel); }
        for (int i = 0; i < ND; i++) {
            const double st = 0 + i / (24.0 * 3600.0 / d->mdt);
            const float zt = (float)interp(st, s);
            for (int j = 0; j < NZ; j++) if (nnz[j] == k) ZT[(size_t)j * ND + i] = zt;
        }
    }
    for (int k = 1; k <= nnq0; k++) {
        snprintf(rel, sizeof rel, "BOUNDE/NQ/NQ%04d.DAT", k);
        Series s;
        if (!read_series(root + rel, s, 0)) { delete d; return fail_io(root + rel); }
        int kl = 0;
        for (int j = 1; j <= NQ; j++) if (k == nnq[j - 1]) kl++;
        for (int i = 0; i < ND; i++) {
            const double st = 0 + i / (24.0 * 3600.0 / d->mdt);
            const float q = (float)interp(st, s);
            for (int j = 0; j < NQ; j++) if (nnq[j] == k) QT[(size_t)j * ND + i] = (double)(q / (float)kl);
        }
    }
    const int K0 = (int)(d->mdt / d->dt);
    const size_t CD = (size_t)C * ND;
    d->qt.assign(CD, 0.0); d->dqt.assign(CD, 0.0); d->zt.assign(CD, 0.0); d->dzt.assign(CD, 0.0);
    for (int i = 0; i < NQ; i++) {
        const int pos = (int)mbq[i] - 1;
        if (pos < 0 || pos >= C) continue;
        for (int jt = 0; jt < ND; jt++) {
            d->qt[(size_t)jt * C + pos] = QT[(size_t)i * ND + jt];
            d->dqt[(size_t)jt * C + pos] = jt != ND - 1 ? (QT[(size_t)i * ND + jt + 1] - QT[(size_t)i * ND + jt]) / K0 : 0.0;
        }
    }
    for (int i = 0; i < NZ; i++) {
        const int pos = (int)mbz[i] - 1;
        if (pos < 0 || pos >= C) continue;
        for (int jt = 0; jt < ND; jt++) {
            d->zt[(size_t)jt * C + pos] = ZT[(size_t)i * ND + jt];
            d->dzt[(size_t)jt * C + pos] = jt != ND - 1 ? (ZT[(size_t)i * ND + jt + 1] - ZT[(size_t)i * ND + jt]) / K0 : 0.0;
        }
    }
    std::vector<double> ZW((size_t)NHQ * NZQ, 0.0), QW((size_t)NHQ * NZQ, 0.0);
    std::vector<int> NHQ1(NZQ, 0);
    for (int k = 1; k <= nnzq0; k++) {
        snprintf(rel, sizeof rel, "BOUNDE/NZQ/NZQ%04d.DAT", k);
        Series s;
        if (!read_series(root + rel, s, 0)) { delete d; return fail_io(root + rel); }
        const int n = (int)s.t.size();
        if (n > NHQ) { delete d; return hb::set_error(HB_E_BADMESH, "deck: %s has %d points, NHQ=%d", rel, n, NHQ); }
        std::vector<double> aqzh0(NZQ, 0.0), aqzh1(NHQ, 0.0);
        for (int i = 0; i < n; i++) {
            for (int j = 0; j < NZQ; j++) {
                if (nnzq[j] != k) continue;
                const int c = (int)mbzq[j] - 1;
                if (c < 0 || c >= C) continue;
                NHQ1[j] = n;
                for (int jj = 0; jj < 4; jj++) {
                    const size_t si = (size_t)c * 4 + jj;
                    if (d->klas[si] == 3) aqzh0[j] = std::fmax(s.t[i] - d->zbc[c], d->hm2) * d->side[si];
                }
                aqzh1[i] += aqzh0[j];
            }
            for (int j = 0; j < NZQ; j++) {
                if (nnzq[j] != k) continue;
                ZW[(size_t)i * NZQ + j] = s.t[i];
                QW[(size_t)i * NZQ + j] = s.v[i] * aqzh0[j] / aqzh1[i];
            }
        }
    }
    d->zw.assign((size_t)C * NHQ, 0.0); d->qw.assign((size_t)C * NHQ, 0.0); d->nhq1.assign(C, 0);
    for (int i = 0; i < NZQ; i++) {
        const int pos = (int)mbzq[i] - 1;
        if (pos < 0 || pos >= C) continue;
        for (int j = 0; j < NHQ; j++) {
            d->zw[(size_t)pos * NHQ + j] = ZW[(size_t)j * NZQ + i];
            d->qw[(size_t)pos * NHQ + j] = QW[(size_t)j * NZQ + i];
        }
        d->nhq1[pos] = NHQ1[i];
    }
    d->bfeat.assign(C, 0.0);
    for (int i = 0; i < d->nwe; i++) {
        const int pos = (int)mbw[i] - 1;
        if (pos >= 0 && pos < C) d->bfeat[pos] = topw[i];
    }
    d->xp = std::move(xp);
    d->yp = std::move(yp);
    d->nap.assign(nap.begin(), nap.end());
    *out = d;
    return HB_OK;
}

extern "C" int hb_deck_mesh(const hb_deck *d, hb_mesh_desc *m) {
    if (!d || !m) return hb::set_error(HB_E_INVALID, "hb_deck_mesh: null argument");
    memset(m, 0, sizeof *m);
    m->cells = d->cells; m->ndays = d->ndays; m->nhq = d->nhq;
    m->steps_per_day = (int)(d->mdt / d->dt);
    m->dt = d->dt; m->hm1 = d->hm1; m->hm2 = d->hm2; m->jl = d->jl;
    m->nac = d->nac.data(); m->klas = d->klas.data();
    m->side = d->side.data(); m->cosf = d->cosf.data(); m->sinf = d->sinf.data();
    m->slcos = d->slcos.data(); m->slsin = d->slsin.data();
    m->zbc = d->zbc.data(); m->zb1 = d->zb1.data(); m->area = d->area.data(); m->fnc = d->fnc.data();
    m->bfeat = d->bfeat.data(); m->nhq1 = d->nhq1.data(); m->zw = d->zw.data(); m->qw = d->qw.data();
    m->qt = d->qt.data(); m->dqt = d->dqt.data(); m->zt = d->zt.data(); m->dzt = d->dzt.data();
    return HB_OK;
}

extern "C" int hb_deck_state(const hb_deck *d, const double **H, const double **U, const double **V,
                             const double **Z, const double **W) {
    if (!d) return hb::set_error(HB_E_INVALID, "hb_deck_state: null deck");
    if (H) *H = d->h.data();
    if (U) *U = d->u.data();
    if (V) *V = d->v.data();
    if (Z) *Z = d->z.data();
    if (W) *W = d->w.data();
    return HB_OK;
}

extern "C" int hb_deck_ntoutput(const hb_deck *d, int32_t *ntoutput) {
    if (!d || !ntoutput) return hb::set_error(HB_E_INVALID, "hb_deck_ntoutput: null argument");
    *ntoutput = d->ntoutput;
    return HB_OK;
}

extern "C" int hb_deck_free(hb_deck *d) {
    delete d;
    return HB_OK;
}

// ---------------------------------------------------------------------------
// OUTPUT writers: the reference's text result files (mesh.cpp:535-839)
// ---------------------------------------------------------------------------
struct hb_output {
    const hb_deck *d = nullptr;
    std::ofstream side, zuv, h2u2v2, tec, timelog;
    bool sides_written = false;
};

namespace {

// Flow direction in radians from the velocity components, quadrant by
// quadrant with pi taken as 3.1416; components below 1e-9 count as zero
// (mesh.cpp:841-875).
double flow_angle(double x, double y) {
    const double pi = 3.1416;
    if (std::fabs(x) < 1e-9) x = 0.0;
    if (std::fabs(y) < 1e-9) y = 0.0;
    if (x * y != 0.0) {
        const double w = std::atan2(std::fabs(y), std::fabs(x));
        if (x * y > 0.0) return x > 0.0 ? w : pi + w;
        return y > 0.0 ? pi - w : 2 * pi - w;
    }
    double f = 0.0;
    if (x == 0.0 && y >= 0.0) f = pi / 2;
    if (x == 0.0 && y < 0.0) f = 3 * pi / 2;
    if (y == 0.0 && x >= 0.0) f = 0.0;
    if (y == 0.0 && x < 0.0) f = pi;
    return f;
}

// the frame header of H2U2V2.OUT and ZUV.OUT
void frame_header(std::ostream &os, int jt2, int kt, double dt) {
    os << " " << std::endl << " " << std::endl;
    os << std::setw(1) << " " << std::setw(3) << "JT=" << std::setw(5) << jt2 << std::setw(2) << " " << "KT="
       << std::setw(5) << kt - 1 << std::setw(2) << " " << "DT=" << std::setw(3) << dt << std::setw(1) << " "
       << "SEC" << std::setw(2) << " " << "T=" << std::setw(2) << 0 << std::setw(1) << "H" << std::setw(2) << " "
       << "NSF=" << std::setw(2) << 0 << "/" << 0 << std::setw(2) << " " << "WEC=" << std::fixed
       << std::setprecision(2) << 0 << "/" << std::setw(2) << " " << "CQL=" << std::fixed << std::setprecision(2) << 0
       << std::setw(2) << " " << "INE=" << std::setw(1) << 0 << std::endl;
}

// one labelled block of per-cell values: 10 per line, an extra break every 100
template <class F>
void value_block(std::ostream &os, const char *label, int n, F value) {
    os << std::setw(5) << " " << std::endl << std::setw(5) << " " << std::setw(3) << label;
    for (int i = 0; i < n; i++) {
        if (i % 10 == 0) os << std::endl << std::setw(5) << " ";
        if (i != 0 && i % 100 == 0) os << std::endl << std::setw(5) << " ";
        os << std::setw(10) << std::fixed << std::setprecision(4) << value(i);
    }
}

// one block of XY-TEC.DAT: 10 values per line
template <class F>
void tec_block(std::ostream &os, int n, bool break_first, F value) {
    for (int i = 0; i < n; i++) {
        if (i % 10 == 0 && (i != 0 || break_first)) os << std::endl;
        os << std::fixed << std::setprecision(4) << value(i) << " ";
    }
}

}  // namespace

extern "C" int hb_output_open(const hb_deck *d, const char *dir, hb_output **out) {
    if (!d || !dir || !out) return hb::set_error(HB_E_INVALID, "hb_output_open: null argument");
    *out = nullptr;
    const std::string base = std::string(dir) + "/";
    auto o = new hb_output();
    o->d = d;
    o->side.open(base + "SIDE.OUT", std::ios::out | std::ofstream::trunc);
    o->zuv.open(base + "ZUV.OUT", std::ios::out | std::ofstream::trunc);
    o->h2u2v2.open(base + "H2U2V2.OUT", std::ios::out | std::ofstream::trunc);
    o->tec.open(base + "XY-TEC.DAT", std::ios::out | std::ofstream::trunc);
    o->timelog.open(base + "TIMELOG.OUT", std::ios::out | std::ofstream::trunc);
    if (!o->side.is_open() || !o->zuv.is_open() || !o->h2u2v2.is_open() || !o->tec.is_open() || !o->timelog.is_open()) {
        delete o;
        return hb::set_error(HB_E_IO, "hb_output_open: cannot create the output files in %s", dir);
    }
    *out = o;
    return HB_OK;
}

extern "C" int hb_output_frame(hb_output *o, int32_t jt, int32_t kt, const double *H, const double *U,
                               const double *V, const double *Z) {
    if (!o || !H || !U || !V || !Z) return hb::set_error(HB_E_INVALID, "hb_output_frame: null argument");
    const hb_deck *d = o->d;
    const int C = d->cells;
    const double HM1 = d->hm1;
    if (jt == 0 && kt == 1 && !o->sides_written) {   // the geometry, with the first frame
        o->sides_written = true;
        const std::vector<double> *per_slot[3] = {&d->cosf, &d->sinf, &d->side};
        const char *names[3] = {"COSF", "SINF", "SIDE"};
        for (int a = 0; a < 3; a++) {
            o->side << names[a] << std::endl;
            for (int i = 0; i < C; i++) {
                o->side << i + 1 << "    ";
                for (int k = 0; k < 4; k++) o->side << (*per_slot[a])[4 * (size_t)i + k] << "     ";
                o->side << std::endl;
            }
        }
        o->side << "AREA" << std::endl;
        for (int i = 0; i < C; i++) o->side << i + 1 << "    " << d->area[i] << std::endl;
    }
    const int jt2 = jt + (kt != 1 ? 1 : 0);
    auto snap = [](double v) { return std::fabs(v) < 1e-9 ? 0.0 : v; };
    auto h2 = [&](int i) { return snap(H[i] <= HM1 ? 0.0 : H[i]); };
    auto u2 = [&](int i) { return snap(H[i] <= HM1 ? 0.0 : U[i]); };
    auto v2 = [&](int i) { return snap(H[i] <= HM1 ? 0.0 : V[i]); };
    auto z2 = [&](int i) { return snap(H[i] <= HM1 ? d->zbc[i] : Z[i]); };
    auto w2 = [&](int i) {   // single precision, as the reference prints it
        float w = 0;
        if (H[i] > HM1) w = std::sqrt(U[i] * U[i] + V[i] * V[i]);
        if (std::fabs(w) < 1e-9f) w = 0;
        return w;
    };
    auto fi = [&](int i) { return H[i] > HM1 ? flow_angle(U[i], V[i]) * (double)57.298 : 0.0; };

    frame_header(o->h2u2v2, jt2, kt, d->dt);
    frame_header(o->zuv, jt2, kt, d->dt);
    value_block(o->h2u2v2, "H2=", C, h2);
    o->h2u2v2 << std::endl;
    value_block(o->h2u2v2, "U2=", C, u2);
    o->h2u2v2 << std::endl;
    value_block(o->h2u2v2, "V2=", C, v2);
    o->h2u2v2 << " " << std::endl;
    value_block(o->zuv, "Z2=", C, z2);
    o->zuv << std::endl;
    value_block(o->zuv, "W2=", C, w2);
    o->zuv << std::endl;
    value_block(o->zuv, "FI=", C, fi);
    o->zuv << " " << std::endl;

    o->timelog << std::fixed << std::setprecision(4) << (double)jt2 / d->ndays << std::endl;

    std::ostream &t = o->tec;
    t << " VARIABLES = \"X\", \"Y\", \"H2\", \"Z2\",\"U2\",\"V2\",\"W2\"" << std::endl;
    t << "ZONE N=" << d->nod << ", E=" << C << ", DATAPACKING=BLOCK, ZONETYPE=FEQUADRILATERAL" << std::endl;
    t << "VARLOCATION=([3-7]=CELLCENTERED)" << std::endl;
    tec_block(t, d->nod, false, [&](int i) { return d->xp[i] + d->ximin; });
    t << std::endl;
    tec_block(t, d->nod, false, [&](int i) { return d->yp[i] + d->yimin; });
    t << std::endl;
    tec_block(t, C, true, [&](int i) { return snap(H[i] <= HM1 ? 0.0 : H[i]); });
    tec_block(t, C, false, z2);
    t << std::endl;
    tec_block(t, C, false, u2);
    t << std::endl;
    tec_block(t, C, false, v2);
    t << std::endl;
    tec_block(t, C, false, w2);
    t << std::endl;
    for (int i = 0; i < C; i++) {
        for (int k = 0; k < 4; k++) t << d->nap[4 * (size_t)i + k] << " ";
        t << std::endl;
    }
    const bool ok = o->side.good() && o->zuv.good() && o->h2u2v2.good() && o->tec.good() && o->timelog.good();
    return ok ? HB_OK : hb::set_error(HB_E_IO, "hb_output_frame: write failed");
}

extern "C" int hb_output_close(hb_output *o) {
    delete o;
    return HB_OK;
}

