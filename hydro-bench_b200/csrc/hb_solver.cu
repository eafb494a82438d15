// hb_solver.cu -- the handle-based path.  The mesh lives on the device in a
// bandwidth-reduced cell order; a step is two kernels chained by programmatic
// dependent launch:
//   flux_kernel    one thread per flux record: an interior edge whose two slots
//                  mirror each other (one Osher evaluation serves both), or a
//                  single slot (CalculateFluxKernel, functors.cu:47-202);
//   update_kernel  one thread per cell: the slot sums in slot order j = 0..3
//                  and the new state (UpdateCellKernel, functors.cu:717-784).
// The state is double-buffered: a step reads buffer (step & 1) and writes the
// other, which is what the reference's two-kernel sequence amounts to.  The
// per-slot flux arrays are written only by the last step of a launch
// sequence, plus every step for the slots whose boundary code leaves some
// fluxes unwritten (those keep their old values, functors.cu:525-565).
//
// A handle may hold a batch of independent scenarios (hb_create_batch).  Their
// cells and records are concatenated, each scenario renumbered on its own, and
// per-CTA segment tables give every CTA one scenario and a record or cell
// range, so one launch pair steps the whole batch.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <queue>
#include <string>
#include <type_traits>
#include <vector>

#include "hb_common.cuh"
#include "hb_physics.cuh"
#include "hydrob200.h"

// ---------------------------------------------------------------------------
// error reporting
// ---------------------------------------------------------------------------
namespace {
thread_local int t_last_status = HB_OK;
thread_local char t_last_msg[512] = "";
}  // namespace

namespace hb {
int set_error(int status, const char *fmt, ...) {
    t_last_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_last_msg, sizeof t_last_msg, fmt, ap);
    va_end(ap);
    return status;
}
}  // namespace hb

extern "C" int hb_last_error(void) { return t_last_status; }
extern "C" const char *hb_last_error_string(void) { return t_last_msg; }
extern "C" const char *hb_status_string(int s) {
    switch (s) {
    case HB_OK: return "ok";
    case HB_E_INVALID: return "invalid argument";
    case HB_E_BADMESH: return "inconsistent mesh";
    case HB_E_CUDA: return "CUDA error";
    case HB_E_NONFINITE: return "non-finite state";
    case HB_E_BARRIER_TIMEOUT: return "grid barrier timeout";
    case HB_E_IO: return "deck file error";
    case HB_E_UNDEFINED_REF: return "slot reached undefined reference behaviour";
    case HB_E_NOMEM: return "out of memory";
    case HB_E_TOO_LARGE: return "size beyond capacity";
    default: return "unknown status";
    }
}

extern "C" void hb_options_default(hb_options *o) {
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->variant = HB_VARIANT_H;
    o->precision = HB_FP64;
    o->device = 0;
    o->renumber = 1;
    o->tile_config = 0;
    o->layout = HB_LAYOUT_EDGE;
    o->tile_cells = 0;
}

#include "hb_handle.hpp"

namespace hb {

// ---------------------------------------------------------------------------
// reverse Cuthill-McKee over the cell adjacency (integer-only; changes no arithmetic)
// ---------------------------------------------------------------------------
std::vector<int32_t> rcm_order(int C, const std::vector<int32_t> &nbr4) {
    std::vector<int> deg(C, 0);
    for (int i = 0; i < C; i++)
        for (int j = 0; j < 4; j++) if (nbr4[4 * i + j] >= 0) deg[i]++;
    std::vector<int32_t> order;
    order.reserve(C);
    std::vector<char> seen(C, 0);
    std::vector<int> cand(C);
    std::iota(cand.begin(), cand.end(), 0);
    std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    auto bfs_last = [&](int start, std::vector<int> &levels) {
        // returns the last node of a BFS from start (a pseudo-peripheral candidate)
        std::queue<int> q;
        std::vector<int> local;
        q.push(start);
        levels[start] = 0;
        int last = start;
        while (!q.empty()) {
            int x = q.front(); q.pop();
            local.push_back(x);
            last = x;
            for (int j = 0; j < 4; j++) {
                int y = nbr4[4 * x + j];
                if (y >= 0 && levels[y] < 0) { levels[y] = levels[x] + 1; q.push(y); }
            }
        }
        for (int x : local) levels[x] = -1;
        return last;
    };
    std::vector<int> levels(C, -1);
    for (int seed : cand) {
        if (seen[seed]) continue;
        int start = bfs_last(bfs_last(seed, levels), levels);
        size_t head = order.size();
        order.push_back(start);
        seen[start] = 1;
        while (head < order.size()) {
            int x = order[head++];
            int nb[4], n = 0;
            for (int j = 0; j < 4; j++) {
                int y = nbr4[4 * x + j];
                if (y >= 0 && !seen[y]) { nb[n++] = y; seen[y] = 1; }
            }
            std::sort(nb, nb + n, [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            for (int q = 0; q < n; q++) order.push_back(nb[q]);
        }
    }
    std::reverse(order.begin(), order.end());
    return order;   // order[new] = old
}

// Tile partition of the tile layout (integer-only; changes no arithmetic).
// Breadth-first balls of up to T cells are grown from the first unassigned
// cell of the reverse Cuthill-McKee order, so consecutive tiles are
// neighbours; then every tile under T/2 cells is merged into the adjacent
// tile it shares most edges with, as long as the sum stays within 5T/4.
// Returns order[new] = old with each tile contiguous, and the tile starts
// (starts.back() == C).
void tile_partition(int C, const std::vector<int32_t> &nbr4, int T, std::vector<int32_t> &order,
                    std::vector<int32_t> &starts) {
    const std::vector<int32_t> seeds = rcm_order(C, nbr4);
    std::vector<int32_t> tile(C, -1);
    std::vector<std::vector<int32_t>> cells;
    for (int seed : seeds) {
        if (tile[seed] >= 0) continue;
        const int t = (int)cells.size();
        cells.emplace_back();
        auto &mem = cells.back();
        mem.push_back(seed);
        tile[seed] = t;
        for (size_t head = 0; head < mem.size() && (int)mem.size() < T; head++) {
            const int x = mem[head];
            for (int j = 0; j < 4 && (int)mem.size() < T; j++) {
                const int y = nbr4[4 * (size_t)x + j];
                if (y >= 0 && tile[y] < 0) { tile[y] = t; mem.push_back(y); }
            }
        }
    }
    const int nt = (int)cells.size();
    std::vector<int> parent(nt);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int x) { while (parent[x] != x) x = parent[x] = parent[parent[x]]; return x; };
    std::vector<int> size(nt);
    for (int t = 0; t < nt; t++) size[t] = (int)cells[t].size();
    const int cap = T + T / 4;
    for (int pass = 0; pass < 3; pass++) {
        std::vector<int> by_size;
        for (int t = 0; t < nt; t++) if (find(t) == t && size[t] < T / 2) by_size.push_back(t);
        std::stable_sort(by_size.begin(), by_size.end(), [&](int a, int b) { return size[a] < size[b]; });
        bool merged = false;
        for (int t : by_size) {
            if (find(t) != t || size[t] >= T / 2) continue;
            std::vector<std::pair<int, int>> shared;   // (neighbour root, shared slots)
            for (int x : cells[t])
                for (int j = 0; j < 4; j++) {
                    const int y = nbr4[4 * (size_t)x + j];
                    if (y < 0) continue;
                    const int r = find(tile[y]);
                    if (r == t) continue;
                    bool found = false;
                    for (auto &e : shared) if (e.first == r) { e.second++; found = true; break; }
                    if (!found) shared.push_back({r, 1});
                }
            int best = -1, best_n = 0;
            for (auto &e : shared)
                if (size[e.first] + size[t] <= cap && (e.second > best_n || (e.second == best_n && e.first < best)))
                    best = e.first, best_n = e.second;
            if (best < 0) continue;
            // the earlier tile keeps its place in the order
            const int keep = std::min(best, t), gone = std::max(best, t);
            cells[keep].insert(cells[keep].end(), cells[gone].begin(), cells[gone].end());
            cells[gone].clear();
            size[keep] += size[gone];
            size[gone] = 0;
            parent[gone] = keep;
            merged = true;
        }
        if (!merged) break;
    }
    order.clear();
    starts.clear();
    for (int t = 0; t < nt; t++) {
        if (find(t) != t) continue;
        starts.push_back((int32_t)order.size());
        order.insert(order.end(), cells[t].begin(), cells[t].end());
    }
    starts.push_back((int32_t)order.size());
}

}  // namespace hb

namespace {

// a and b have the same bit pattern (so -0.0 differs from +0.0)
bool same_bits(double a, double b) {
    uint64_t x, y;
    std::memcpy(&x, &a, sizeof x);
    std::memcpy(&y, &b, sizeof y);
    return x == y;
}

// Host image of the device mesh of every scenario, concatenated.
template <class A>
struct HostMesh {
    using R = typename A::real;
    using L = typename A::level;
    std::vector<L> zbc;
    std::vector<R> fnc, area, side4;
    std::vector<uint8_t> cmask;
    std::vector<int4> rix;
    std::vector<uint8_t> rmeta;
    std::vector<R> rgeo;
    std::vector<int32_t> bcell;               // global table row, -1 = none
    // one entry per table row: the row's values for each interval of its scenario
    std::vector<std::vector<R>> qt, dqt;
    std::vector<std::vector<L>> zt, dzt;
    std::vector<L> top;
    std::vector<int32_t> nhq1;
    std::vector<std::vector<L>> zw;
    std::vector<std::vector<R>> qw;
};

// Validates one scenario's mesh and appends it (renumbered) to hm.
template <class A>
int append_scenario(const hb_mesh_desc *md, int scn, const hb_options &opt, hb::Scenario &sc, HostMesh<A> &hm) {
    using R = typename A::real;
    using L = typename A::level;
    if (md->cells <= 0 || md->ndays <= 0 || md->steps_per_day < 2 || md->nhq < 0)
        return hb::set_error(HB_E_INVALID, "mesh: cells=%d ndays=%d steps_per_day=%d", md->cells, md->ndays,
                             md->steps_per_day);
    const double *need[] = {md->nac, md->klas, md->side, md->cosf, md->sinf, md->zbc, md->area, md->fnc,
                            md->bfeat, md->qt, md->dqt, md->zt, md->dzt};
    for (const double *p : need) if (!p) return hb::set_error(HB_E_INVALID, "mesh: missing array");
    if (md->nhq > 0 && (!md->zw || !md->qw || !md->nhq1)) return hb::set_error(HB_E_INVALID, "mesh: missing rating tables");
    const int C = md->cells;
    const size_t S = 4 * (size_t)C;
    sc.cells = C;
    sc.cell0 = (int)hm.zbc.size();
    sc.ndays = md->ndays; sc.nhq = md->nhq;
    sc.steps_per_day = md->steps_per_day; sc.per_day = md->steps_per_day - 1;
    sc.dt = md->dt; sc.hm1 = md->hm1; sc.hm2 = md->hm2; sc.jl = md->jl;
    // neighbour lists in input order, for the renumbering
    std::vector<int32_t> nbr_old(S, -1);
    for (size_t s = 0; s < S; s++) {
        const int nc = (int)(md->nac[s] - 1.0);
        if (nc != -1 && (nc < 0 || nc >= C)) return hb::set_error(HB_E_BADMESH, "NAC[%zu] = %g out of range", s, md->nac[s]);
        nbr_old[s] = nc;
    }
    std::vector<int32_t> starts;
    if (opt.layout == HB_LAYOUT_TILE) {
        hb::tile_partition(C, nbr_old, opt.tile_cells > 0 ? opt.tile_cells : 256, sc.perm, starts);
    } else {
        if (opt.renumber) sc.perm = hb::rcm_order(C, nbr_old);
        else { sc.perm.resize(C); std::iota(sc.perm.begin(), sc.perm.end(), 0); }
        starts = {0, C};
    }
    std::vector<int32_t> tile_of(C);
    for (size_t t = 0; t + 1 < starts.size(); t++)
        for (int i = starts[t]; i < starts[t + 1]; i++) tile_of[i] = (int32_t)t;
    sc.inv.assign(C, -1);
    for (int i = 0; i < C; i++) sc.inv[sc.perm[i]] = i;
    sc.klas_orig.assign(md->klas, md->klas + S);
    const auto &perm = sc.perm;
    const auto &inv = sc.inv;
    const int c0 = sc.cell0;
    for (int i = 0; i < C; i++) {
        hm.zbc.push_back((L)md->zbc[perm[i]]);
        hm.fnc.push_back((R)md->fnc[perm[i]]);
        hm.area.push_back((R)md->area[perm[i]]);
        for (int j = 0; j < 4; j++) hm.side4.push_back((R)md->side[4 * (size_t)perm[i] + j]);
    }
    // real slots: everything except a zero-length slot without neighbour and code 0
    std::vector<int32_t> nbr4(S, -1);
    std::vector<uint8_t> meta4(S, 0);
    std::vector<char> real4(S, 0);
    std::vector<char> needs_table(C, 0);
    for (int i = 0; i < C; i++) {
        const int old = perm[i];
        for (int j = 0; j < 4; j++) {
            const size_t so = 4 * (size_t)old + j, sn = 4 * (size_t)i + j;
            const int nc_old = nbr_old[so];
            const int8_t code = hb::klas_code(md->klas[so]);
            uint8_t mt = (uint8_t)code;
            if (nc_old != -1) {
                nbr4[sn] = inv[nc_old];
                mt |= hb::META_HAS_NB;
                if (old < nc_old) mt |= hb::META_OWN_FIRST;
            }
            meta4[sn] = mt;
            real4[sn] = !(md->side[so] == 0.0 && md->cosf[so] == 0.0 && md->sinf[so] == 0.0 && nc_old == -1 &&
                          code == hb::CODE_ZERO);
            if (code == hb::CODE_K10 || code == hb::CODE_K1 || code == hb::CODE_K3 || code == hb::CODE_K6 ||
                code == hb::CODE_K7)
                needs_table[i] = 1;
        }
    }
    for (int i = 0; i < C; i++) {
        uint8_t cm = 0;
        for (int j = 0; j < 4; j++)
            if (real4[4 * (size_t)i + j]) cm |= (uint8_t)(1u << j);
        hm.cmask.push_back(cm);
    }
    // records, tile by tile: exact mirror pairs inside the tile first, then
    // every other real slot of the tile's cells
    sc.rec0 = (int)hm.rix.size();
    std::vector<char> paired(S, 0);
    auto slot_of = [&](int i, int j) { return 4 * (size_t)perm[i] + j; };   // reference slot of device slot
    auto push = [&](int a, int b, size_t sa, long long sb, uint8_t mt, size_t so) {
        hm.rix.push_back(make_int4(c0 + a, b < 0 ? -1 : c0 + b, (int)(4 * (size_t)c0 + sa),
                                   sb < 0 ? -1 : (int)(4 * (size_t)c0 + sb)));
        hm.rmeta.push_back(mt);
        hm.rgeo.push_back((R)md->cosf[so]); hm.rgeo.push_back((R)md->sinf[so]);
        hm.rgeo.push_back((R)md->side[so]); hm.rgeo.push_back(R(0));
    };
    sc.slot_index.assign(S, -1);
    sc.npairs = 0;
    sc.tiles.clear();
    for (size_t t = 0; t + 1 < starts.size(); t++) {
        hb::TileDesc td{scn, c0 + starts[t], starts[t + 1] - starts[t], (int)hm.rix.size(), 0, 0};
        for (int i = starts[t]; i < starts[t + 1]; i++) {
            for (int j = 0; j < 4; j++) {
                const size_t sn = 4 * (size_t)i + j;
                if (!real4[sn] || paired[sn] || (meta4[sn] & hb::META_CODE) != hb::CODE_ZERO || nbr4[sn] < 0) continue;
                if (!(meta4[sn] & hb::META_OWN_FIRST)) continue;      // the pair is listed from its lower-numbered side
                const int nb = nbr4[sn];
                if (tile_of[nb] != (int32_t)t) continue;
                int jb = -1;
                for (int q = 0; q < 4; q++)
                    if (nbr4[4 * (size_t)nb + q] == i && !paired[4 * (size_t)nb + q]) { jb = q; break; }
                if (jb < 0) continue;
                const size_t sb = 4 * (size_t)nb + jb;
                const size_t oa = slot_of(i, j), ob = slot_of(nb, jb);
                // the two slots must see one edge: code 0 both, negated normal, same
                // length, bit for bit (a zero component must have the opposite sign
                // too: the mirrored side is evaluated with the negated normal, and a
                // wrongly signed zero changes the sign of zero results)
                if ((meta4[sb] & hb::META_CODE) != hb::CODE_ZERO || !real4[sb] || !same_bits(md->cosf[ob], -md->cosf[oa]) ||
                    !same_bits(md->sinf[ob], -md->sinf[oa]) || !same_bits(md->side[ob], md->side[oa]))
                    continue;
                paired[sn] = paired[sb] = 1;
                push(i, nb, sn, (long long)sb, meta4[sn], oa);
                td.npairs++;
            }
        }
        for (int i = starts[t]; i < starts[t + 1]; i++) {
            for (int j = 0; j < 4; j++) {
                const size_t sn = 4 * (size_t)i + j;
                if (!real4[sn] || paired[sn]) continue;
                sc.slot_index[sn] = (int32_t)hm.rix.size();
                push(i, nbr4[sn], sn, -1, meta4[sn], slot_of(i, j));
                td.nsingles++;
            }
        }
        sc.npairs += td.npairs;
        sc.tiles.push_back(td);
    }
    sc.nrecords = (int)hm.rix.size() - sc.rec0;
    // boundary table rows of the cells that need them
    const int NHQ = std::max(md->nhq, 0);
    for (int i = 0; i < C; i++) {
        if (!needs_table[i]) { hm.bcell.push_back(-1); continue; }
        hm.bcell.push_back((int32_t)hm.top.size());
        const int old = perm[i];
        std::vector<R> q(md->ndays), dq(md->ndays), w(NHQ);
        std::vector<L> z(md->ndays), dz(md->ndays), zw(NHQ);
        for (int d = 0; d < md->ndays; d++) {
            const size_t t = (size_t)d * C + old;
            q[d] = (R)md->qt[t]; dq[d] = (R)md->dqt[t]; z[d] = (L)md->zt[t]; dz[d] = (L)md->dzt[t];
        }
        for (int k = 0; k < NHQ; k++) {
            zw[k] = (L)md->zw[(size_t)old * NHQ + k];
            w[k] = (R)md->qw[(size_t)old * NHQ + k];
        }
        hm.qt.push_back(q); hm.dqt.push_back(dq); hm.zt.push_back(z); hm.dzt.push_back(dz);
        hm.top.push_back((L)md->bfeat[old]);
        hm.nhq1.push_back(NHQ > 0 ? md->nhq1[old] : 0);
        hm.zw.push_back(zw); hm.qw.push_back(w);
    }
    return HB_OK;
}

// Segment tables: CTAs of `threads` records (flux) or UPDATE_THREADS cells
// (update), none straddling two scenarios or the pair/single boundary.
std::vector<int4> flux_segments(const std::vector<hb::Scenario> &scn, int threads) {
    std::vector<int4> seg;
    for (int s = 0; s < (int)scn.size(); s++)
        for (const hb::TileDesc &td : scn[s].tiles) {
            for (int b = 0; b < td.npairs; b += threads)
                seg.push_back(make_int4(s, td.rec0 + b, std::min(threads, td.npairs - b), 1));
            for (int b = 0; b < td.nsingles; b += threads)
                seg.push_back(make_int4(s, td.rec0 + td.npairs + b, std::min(threads, td.nsingles - b), 0));
        }
    return seg;
}
std::vector<int4> update_segments(const std::vector<hb::Scenario> &scn) {
    std::vector<int4> seg;
    for (int s = 0; s < (int)scn.size(); s++)
        for (int b = 0; b < scn[s].cells; b += hb::UPDATE_THREADS)
            seg.push_back(make_int4(s, scn[s].cell0 + b, std::min(hb::UPDATE_THREADS, scn[s].cells - b), 0));
    return seg;
}

int thread_slot(int threads) { return threads == 64 ? 0 : threads == 128 ? 1 : 2; }

template <class A>
int build_device_mesh(hb_handle *h, const hb_mesh_desc *mds, int n, hb::DevMesh<A> &m) {
    using R = typename A::real;
    using L = typename A::level;
    HostMesh<A> hm;
    // tile layout: tiles of h->tile_cells cells; with the balanced default
    // (tile_waves > 0) the size grows until the tiles fill at most tile_waves
    // whole waves of tile_slots resident CTAs (a tile count just above a wave
    // leaves most SMs idle while a few run the extra tiles)
    hb_options opt = h->opt;
    for (int pass = 0;; pass++) {
        opt.tile_cells = h->tile_cells;
        hm = HostMesh<A>();
        h->scn.assign(n, hb::Scenario());
        for (int s = 0; s < n; s++) {
            const int st = append_scenario<A>(&mds[s], s, opt, h->scn[s], hm);
            if (st != HB_OK) return n > 1 ? hb::set_error(st, "scenario %d: %s", s, hb_last_error_string()) : st;
        }
        if (opt.layout != HB_LAYOUT_TILE || h->tile_waves <= 0 || pass == 3) break;
        long long tiles = 0;
        for (const auto &sc : h->scn) tiles += (long long)sc.tiles.size();
        const long long cap = (long long)h->tile_waves * h->tile_slots;
        if (tiles <= cap || h->tile_cells >= 1024) break;
        h->tile_cells = std::min(1024, (int)((h->tile_cells * tiles + cap - 1) / cap) + 1);
    }
    const int C = (int)hm.zbc.size();
    h->C = C;
    h->max_cells = 0;
    for (const auto &sc : h->scn) h->max_cells = std::max(h->max_cells, sc.cells);
    const hb::Scenario &s0 = h->scn[0];
    m.C = C;
    m.per_day = s0.per_day; m.ndays = s0.ndays;
    m.hm1 = s0.hm1; m.hm2 = s0.hm2; m.jl = s0.jl; m.dt = s0.dt;
    m.npairs = s0.npairs;                 // a single mesh's records: [0, npairs) pairs
    m.nrecords = (int)hm.rix.size();
    // boundary tables: [day][row] over the longest scenario; a scenario's rows
    // repeat its last interval beyond its own tables (never read: step_index clamps)
    const int NB = (int)hm.top.size();
    int ND = 1, NHQ = 0;
    for (const auto &sc : h->scn) { ND = std::max(ND, sc.ndays); NHQ = std::max(NHQ, sc.nhq); }
    std::vector<R> bqt((size_t)ND * NB), bdqt((size_t)ND * NB), bqw((size_t)(NB + 1) * NHQ, R(0));
    std::vector<L> bzt((size_t)ND * NB), bdzt((size_t)ND * NB), bzw((size_t)(NB + 1) * NHQ, L(0));
    for (int r = 0; r < NB; r++) {
        const int nd = (int)hm.qt[r].size();
        for (int d = 0; d < ND; d++) {
            const int dd = std::min(d, nd - 1);
            bqt[(size_t)d * NB + r] = hm.qt[r][dd]; bdqt[(size_t)d * NB + r] = hm.dqt[r][dd];
            bzt[(size_t)d * NB + r] = hm.zt[r][dd]; bdzt[(size_t)d * NB + r] = hm.dzt[r][dd];
        }
        for (size_t k = 0; k < hm.zw[r].size(); k++) {
            bzw[(size_t)r * NHQ + k] = hm.zw[r][k];
            bqw[(size_t)r * NHQ + k] = hm.qw[r][k];
        }
    }
    m.nb = NB;
    m.nhq = NHQ;
    int32_t *ip;
    uint8_t *up;
    R *rp;
    L *lp;
    TRY(dev_upload(h, &lp, hm.zbc)); m.zbc = lp;
    TRY(dev_upload(h, &rp, hm.fnc)); m.fnc = rp;
    R *area_d = nullptr, *side_d = nullptr;
    TRY(dev_upload(h, &area_d, hm.area));
    TRY(dev_upload(h, &side_d, hm.side4));   // [4C], for the per-cell setup only
    TRY(dev_upload(h, &up, hm.cmask)); m.cmask = up;
    {
        int4 *ixp;
        TRY(dev_upload(h, &ixp, hm.rix)); m.rix = ixp;
        TRY(dev_upload(h, &rp, hm.rgeo)); m.rgeo = rp;
    }
    TRY(dev_upload(h, &up, hm.rmeta)); m.rmeta = up;
    TRY(dev_upload(h, &ip, hm.bcell)); m.bcell = ip;
    TRY(dev_upload(h, &rp, bqt)); m.bqt = rp;
    TRY(dev_upload(h, &rp, bdqt)); m.bdqt = rp;
    TRY(dev_upload(h, &lp, bzt)); m.bzt = lp;
    TRY(dev_upload(h, &lp, bdzt)); m.bdzt = lp;
    TRY(dev_upload(h, &lp, hm.top)); m.btop = lp;
    TRY(dev_upload(h, &ip, hm.nhq1)); m.bnhq1 = ip;
    TRY(dev_upload(h, &lp, bzw)); m.bzw = lp;
    TRY(dev_upload(h, &rp, bqw)); m.bqw = rp;
    const size_t S = 4 * (size_t)C;
    for (int b = 0; b < 2; b++) TRY(dev_alloc(h, &m.S[b], 4 * (size_t)C));
    TRY(dev_alloc(h, &m.slotw, 16 * (size_t)C));
    TRY(dev_alloc(h, &m.W, C));
    TRY(dev_alloc(h, &m.f0, S)); TRY(dev_alloc(h, &m.f1, S));
    TRY(dev_alloc(h, &m.f2, S)); TRY(dev_alloc(h, &m.f3, S));
    R *dta = nullptr, *sidex = nullptr;
    TRY(dev_alloc(h, &dta, C));
    TRY(dev_alloc(h, &sidex, C));
    for (const auto &sc : h->scn) {
        const int blocks = (sc.cells + 255) / 256;
        const size_t c0 = sc.cell0;
        if (h->opt.variant == HB_VARIANT_F)
            hb::setup_cells_kernel<A, 1><<<blocks, 256>>>(sc.cells, sc.dt, area_d + c0, side_d + 4 * c0, dta + c0, sidex + c0);
        else
            hb::setup_cells_kernel<A, 0><<<blocks, 256>>>(sc.cells, sc.dt, area_d + c0, side_d + 4 * c0, dta + c0, sidex + c0);
        HB_CUDA_RET(cudaGetLastError());
    }
    HB_CUDA_RET(cudaDeviceSynchronize());
    m.dta = dta;
    m.sidex = sidex;
    m.err = h->d_err;
    m.step_ctr = h->d_ctr;
    // scenario table and segment tables
    std::vector<hb::ScnParams> sp;
    for (const auto &sc : h->scn)
        sp.push_back(hb::ScnParams{sc.hm1, sc.hm2, sc.jl, sc.dt, sc.per_day, sc.ndays, sc.cell0, sc.cells});
    hb::ScnParams *spd;
    TRY(dev_upload(h, &spd, sp)); m.scn = spd;
    m.nscen = n;
    const int tsizes[3] = {64, 128, 256};
    for (int t = 0; t < 3; t++) {
        const std::vector<int4> seg = flux_segments(h->scn, tsizes[t]);
        h->nfseg[t] = (int)seg.size();
        TRY(dev_upload(h, &h->d_fseg[t], seg));
    }
    {
        const std::vector<int4> seg = update_segments(h->scn);
        h->nuseg = (int)seg.size();
        TRY(dev_upload(h, &h->d_useg, seg));
    }
    m.fseg = h->d_fseg[1];
    m.useg = h->d_useg;
    m.rev_flux = 1;     // single mesh: flux CTAs last range first, cells first range first
    m.rev_update = 1;   // batches: flux segments in order, cells reversed
    {
        std::vector<hb::TileDesc> tiles;
        m.max_tile_cells = 1;
        m.max_tile_pairs = 1;
        for (const auto &sc : h->scn)
            for (const auto &td : sc.tiles) {
                tiles.push_back(td);
                m.max_tile_cells = std::max(m.max_tile_cells, td.cells);
                m.max_tile_pairs = std::max(m.max_tile_pairs, td.npairs);
            }
        m.ntiles = (int)tiles.size();
        hb::TileDesc *tp;
        TRY(dev_upload(h, &tp, tiles));
        m.tiles = tp;
    }
    // scenario permutations on the device, for the staging kernels
    std::vector<int32_t> perms;
    for (const auto &sc : h->scn) perms.insert(perms.end(), sc.perm.begin(), sc.perm.end());
    TRY(dev_upload(h, &h->d_perm, perms));
    TRY(dev_alloc(h, &h->d_stage, 5 * (size_t)h->max_cells));
    return HB_OK;
}

// The counter tick after a step sequence, chained to it by programmatic
// dependent launch.
int launch_tick(hb_handle *h, int n, cudaStream_t st) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(1);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    HB_CUDA_RET(cudaLaunchKernelEx(&cfg, hb::tick_kernel, h->d_ctr, n));
    return HB_OK;
}

template <class A, int VARIANT, bool SEG>
int launch_steps_t(hb_handle *h, hb::DevMesh<A> m, int n, cudaStream_t st) {
    // Programmatic dependent launch: each kernel may start while its predecessor
    // drains and waits in cudaGridDependencySynchronize for its results.
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg_u{};
    cfg_u.gridDim = SEG ? dim3((unsigned)std::max(1, h->nuseg))
                        : dim3((unsigned)std::max(1, (h->C + hb::UPDATE_THREADS - 1) / hb::UPDATE_THREADS));
    cfg_u.blockDim = dim3(hb::UPDATE_THREADS);
    cfg_u.stream = st;
    cfg_u.attrs = attr;
    cfg_u.numAttrs = 1;
    auto go = [&](auto flux, int threads, auto update) -> int {
        cudaLaunchConfig_t cfg_f = cfg_u;
        const int ts = thread_slot(threads);
        m.fseg = h->d_fseg[ts];
        cfg_f.gridDim = SEG ? dim3((unsigned)std::max(1, h->nfseg[ts]))
                            : dim3((unsigned)std::max(1, (m.nrecords + threads - 1) / threads));
        cfg_f.blockDim = dim3(threads);
        for (int k = 0; k < n; k++) {
            HB_CUDA_RET(cudaLaunchKernelEx(&cfg_f, flux, m, k, (int)(k == n - 1)));
            HB_CUDA_RET(cudaLaunchKernelEx(&cfg_u, update, m, k, (int)(k == n - 1)));
        }
        return HB_OK;
    };
    int rc;
    using namespace hb;
    switch (h->launch_config) {
    case 0: rc = go(flux_kernel<A, VARIANT, 128, 7, SEG>, 128, update_kernel<A, VARIANT, 8, SEG>); break;
    case 1: rc = go(flux_kernel<A, VARIANT, 128, 6, SEG>, 128, update_kernel<A, VARIANT, 8, SEG>); break;
    case 2: rc = go(flux_kernel<A, VARIANT, 128, 8, SEG>, 128, update_kernel<A, VARIANT, 8, SEG>); break;
    case 3: rc = go(flux_kernel<A, VARIANT, 256, 3, SEG>, 256, update_kernel<A, VARIANT, 6, SEG>); break;
    case 4: rc = go(flux_kernel<A, VARIANT, 256, 4, SEG>, 256, update_kernel<A, VARIANT, 8, SEG>); break;
    case 5: rc = go(flux_kernel<A, VARIANT, 128, 7, SEG>, 128, update_kernel<A, VARIANT, 6, SEG>); break;
    case 6: rc = go(flux_kernel<A, VARIANT, 256, 2, SEG>, 256, update_kernel<A, VARIANT, 6, SEG>); break;
    case 7: rc = go(flux_kernel<A, VARIANT, 64, 12, SEG>, 64, update_kernel<A, VARIANT, 8, SEG>); break;
    case 14: rc = go(flux_kernel<A, VARIANT, 128, 6, SEG>, 128, update_kernel<A, VARIANT, 6, SEG>); break;
    case 15: rc = go(flux_kernel<A, VARIANT, 128, 6, SEG>, 128, update_kernel<A, VARIANT, 9, SEG>); break;
    case 16: rc = go(flux_kernel<A, VARIANT, 128, 7, SEG>, 128, update_kernel<A, VARIANT, 9, SEG>); break;
    default: return hb::set_error(HB_E_INVALID, "launch shape %d is not an edge-layout shape", h->launch_config + 1);
    }
    if (rc != HB_OK) return rc;
    return launch_tick(h, n, st);
}

// Persistent handles: the whole sequence as cooperative launches of
// persistent_kernel (128 threads, 6 CTAs per SM), as many CTAs as are
// resident at once, each launch preceded by zeroing its barrier words.
// A launch takes at most PERSIST_MAX_STEPS steps, and fewer where its grid
// is larger: every step adds 2 x grid arrivals to the 32-bit arrival count,
// which must stay below 2^32 (phantom arrivals included) so that no barrier
// target wraps.  Longer sequences take several launches; the extra flux
// writes at the end of each launch leave the same final fluxes.
constexpr int PERSIST_THREADS = 128, PERSIST_MINB = 6, PERSIST_MAX_STEPS = 1 << 20;

// Steps one cooperative launch of `grid` CTAs may take (>= 1).
inline int persist_steps_per_launch(unsigned grid, unsigned phantom) {
    const unsigned long long room = 0xFFFFFFFFull - phantom;
    const unsigned long long k = room / (2ull * std::max(1u, grid) + 1ull);
    return (int)std::max(1ull, std::min(k, (unsigned long long)PERSIST_MAX_STEPS));
}

template <class A, int VARIANT, bool SEG>
int launch_persistent_t(hb_handle *h, hb::DevMesh<A> m, int n, cudaStream_t st) {
    auto kernel = hb::persistent_kernel<A, VARIANT, PERSIST_THREADS, PERSIST_MINB, SEG>;
    const int ts = thread_slot(PERSIST_THREADS);
    m.fseg = h->d_fseg[ts];
    const int nflux = SEG ? h->nfseg[ts] : (m.nrecords + PERSIST_THREADS - 1) / PERSIST_THREADS;
    const int ncell = SEG ? h->nuseg : (h->C + hb::UPDATE_THREADS - 1) / hb::UPDATE_THREADS;
    if (h->persist_blocks == 0) {
        int per_sm = 0, sms = 0;
        HB_CUDA_RET(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, PERSIST_THREADS, 0));
        HB_CUDA_RET(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->opt.device));
        if (per_sm < 1) return hb::set_error(HB_E_CUDA, "persistent kernel: no CTA fits on an SM");
        h->persist_blocks = per_sm * sms;
    }
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)std::max(1, std::min(h->persist_blocks, std::max(nflux, ncell))));
    cfg.blockDim = dim3(PERSIST_THREADS);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int kmax = persist_steps_per_launch(cfg.gridDim.x, h->barrier_phantom);
    for (int done = 0; done < n;) {
        const int k = std::min(n - done, kmax);
        HB_CUDA_RET(cudaMemsetAsync(h->d_bar, 0, 2 * sizeof(unsigned), st));
        HB_CUDA_RET(cudaLaunchKernelEx(&cfg, kernel, m, k, nflux, ncell, h->d_bar, h->barrier_phantom,
                                       h->barrier_limit_ns));
        // the step counter advances per launch: the next launch's steps follow on
        TRY(launch_tick(h, k, st));
        done += k;
    }
    return HB_OK;
}

int enqueue_steps(hb_handle *h, int n, cudaStream_t st) {
    if (n <= 0) return HB_OK;
    const bool f = h->opt.variant == HB_VARIANT_F;
    const bool seg = h->segmented();
    const bool tiles = h->opt.layout == HB_LAYOUT_TILE;
    return h->with_mesh([&](auto &m) {
        using A = typename std::remove_reference<decltype(m)>::type::Policy;
        if (tiles) return hb_tiles_launch(h, n, st);
        if (h->opt.persistent) {
            if (seg) return f ? launch_persistent_t<A, 1, true>(h, m, n, st) : launch_persistent_t<A, 0, true>(h, m, n, st);
            return f ? launch_persistent_t<A, 1, false>(h, m, n, st) : launch_persistent_t<A, 0, false>(h, m, n, st);
        }
        if (seg) return f ? launch_steps_t<A, 1, true>(h, m, n, st) : launch_steps_t<A, 0, true>(h, m, n, st);
        return f ? launch_steps_t<A, 1, false>(h, m, n, st) : launch_steps_t<A, 0, false>(h, m, n, st);
    });
}

int default_config(int layout) {
    return layout == HB_LAYOUT_TILE ? hb::DEFAULT_TILE_CONFIG : hb::DEFAULT_EDGE_CONFIG;
}

// launch shape index of tile_config (0 = the layout's default), or -1
int config_for(int layout, int tile_config) {
    if (tile_config == 0) return default_config(layout);
    if (tile_config < 0 || tile_config > hb::N_LAUNCH_CONFIGS) return -1;
    return hb::LAUNCH_CONFIGS[tile_config - 1].layout == layout ? tile_config - 1 : -1;
}

int check_range(hb_handle *h, long long n) {
    const long long limit = h->step_limit();
    if (h->steps_done + n > limit)
        return hb::set_error(HB_E_INVALID, "step %lld..%lld beyond the boundary tables (%lld steps)", h->steps_done,
                             h->steps_done + n, limit);
    return HB_OK;
}

}  // namespace

int hb_enqueue_steps(hb_handle *h, int n, cudaStream_t st) { return enqueue_steps(h, n, st); }

bool hb_steps_take_mesh(const hb_handle *h) {
    return h->opt.precision == HB_FP64 && h->opt.layout == HB_LAYOUT_EDGE && !h->opt.persistent && !h->segmented();
}

int hb_enqueue_steps_mesh(hb_handle *h, const hb::DevMesh<hb::F64Exact> &m, int n, cudaStream_t st) {
    if (!hb_steps_take_mesh(h)) return hb::set_error(HB_E_INVALID, "steps from a mesh copy: fp64 edge-layout single meshes only");
    if (n <= 0) return HB_OK;
    return h->opt.variant == HB_VARIANT_F ? launch_steps_t<hb::F64Exact, 1, false>(h, m, n, st)
                                          : launch_steps_t<hb::F64Exact, 0, false>(h, m, n, st);
}
int hb_launch_tick(hb_handle *h, int n, cudaStream_t st) { return launch_tick(h, n, st); }
int hb_check_range(hb_handle *h, long long n) { return check_range(h, n); }

int hb_forward_step_into(hb_handle *h, long long t0, int k, const double *in, double *out, double *terms,
                         double *coef, int write_flux, cudaStream_t st) {
    hb::DevMesh<hb::F64Exact> m = h->m64;
    const int par = (int)((t0 + k) & 1);
    m.S[par] = const_cast<double *>(in);
    m.S[par ^ 1] = out;
    m.slotw = terms;
    m.ucoef = coef;
    // programmatic dependent launch, as in the step sequence (launch_steps_t)
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3((unsigned)((m.nrecords + 127) / 128));
    cfg.blockDim = dim3(128);
    HB_CUDA_RET(cudaLaunchKernelEx(&cfg, hb::flux_kernel<hb::F64Exact, 0, 128, 6, false, false>, m, k, write_flux));
    cfg.gridDim = dim3((unsigned)((m.C + hb::UPDATE_THREADS - 1) / hb::UPDATE_THREADS));
    cfg.blockDim = dim3(hb::UPDATE_THREADS);
    HB_CUDA_RET(cudaLaunchKernelEx(&cfg, hb::update_kernel<hb::F64Exact, 0, 6, false, true>, m, k, write_flux));
    return HB_OK;
}

namespace {

int check_scenario(hb_handle *h, int s) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    if (s < 0 || s >= (int)h->scn.size())
        return hb::set_error(HB_E_INVALID, "scenario %d outside 0..%d", s, (int)h->scn.size() - 1);
    return HB_OK;
}

}  // namespace

extern "C" int hb_launch_shapes(int32_t *layout, int32_t *threads, int32_t *min_blocks, int32_t capacity) {
    for (int i = 0; i < hb::N_LAUNCH_CONFIGS && i < capacity; i++) {
        if (layout) layout[i] = hb::LAUNCH_CONFIGS[i].layout;
        if (threads) threads[i] = hb::LAUNCH_CONFIGS[i].threads;
        if (min_blocks) min_blocks[i] = hb::LAUNCH_CONFIGS[i].min_blocks * 100 + hb::LAUNCH_CONFIGS[i].update_min_blocks;
    }
    return hb::N_LAUNCH_CONFIGS;
}

extern "C" int hb_tile_configs(int32_t *threads, int32_t *min_blocks, int32_t capacity) {
    for (int i = 0; i < hb::N_LAUNCH_CONFIGS && i < capacity; i++) {
        if (threads) threads[i] = hb::LAUNCH_CONFIGS[i].threads;
        if (min_blocks) min_blocks[i] = hb::LAUNCH_CONFIGS[i].min_blocks * 100 + hb::LAUNCH_CONFIGS[i].update_min_blocks;
    }
    return hb::N_LAUNCH_CONFIGS;
}

extern "C" int hb_create_batch(const hb_mesh_desc *meshes, int32_t n, const hb_options *opt_in, hb_handle **out) {
    if (!meshes || !out || n <= 0) return hb::set_error(HB_E_INVALID, "hb_create_batch: bad argument");
    *out = nullptr;
    hb_options opt;
    if (opt_in) opt = *opt_in; else hb_options_default(&opt);
    if (opt.precision != HB_FP64 && opt.precision != HB_FP32 && opt.precision != HB_SPLIT)
        return hb::set_error(HB_E_INVALID, "hb_create: precision %d not available on this path", opt.precision);
    if (opt.layout != HB_LAYOUT_EDGE && opt.layout != HB_LAYOUT_TILE)
        return hb::set_error(HB_E_INVALID, "hb_create: layout %d", opt.layout);
    if (opt.tile_cells < 0 || opt.tile_cells > 1024)   // 5/4 x 1024 fp64 cells: 160 KB of shared memory
        return hb::set_error(HB_E_INVALID, "hb_create: tile_cells %d outside 0..1024", opt.tile_cells);
    if (config_for(opt.layout, opt.tile_config) < 0)
        return hb::set_error(HB_E_INVALID, "hb_create: tile_config %d is no shape of layout %d", opt.tile_config, opt.layout);
    if (opt.persistent != 0 && opt.persistent != 1)
        return hb::set_error(HB_E_INVALID, "hb_create: persistent %d", opt.persistent);
    if (opt.persistent && (opt.layout != HB_LAYOUT_EDGE || config_for(opt.layout, opt.tile_config) != hb::DEFAULT_EDGE_CONFIG))
        return hb::set_error(HB_E_INVALID, "hb_create: a persistent handle takes the edge layout's default launch shape");
    long long total = 0;
    for (int s = 0; s < n; s++) total += std::max(meshes[s].cells, 0);
    if (total > (1 << 29)) return hb::set_error(HB_E_TOO_LARGE, "hb_create: %lld cells", total);
    HB_CUDA_RET(cudaSetDevice(opt.device));
    auto h = new hb_handle();
    h->opt = opt;
    h->launch_config = config_for(opt.layout, opt.tile_config);
    h->tile_cells = opt.tile_cells > 0 ? opt.tile_cells : 256;
    if (opt.layout == HB_LAYOUT_TILE && opt.tile_cells == 0 && opt.precision != HB_FP64) {
        // balanced default (fp32 state): about 512 cells per tile, adjusted so
        // the tiles fill whole waves of the launch shape's resident CTAs.  The
        // fp64 tile kernel keeps 256: its 128 bytes of slot terms per cell make
        // its occupancy step with the tile size, and smaller balanced tiles
        // measured slower there.
        int sms = 0, per_sm = 0;
        cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, opt.device);
        int rs = e == cudaSuccess ? hb_tiles_resident(h, h->launch_config, 512, &per_sm) : HB_E_CUDA;
        if (rs != HB_OK || sms <= 0 || per_sm <= 0) {
            delete h;
            return rs != HB_OK ? rs : hb::set_error(HB_E_CUDA, "hb_create: no tile CTA fits on an SM");
        }
        h->tile_slots = sms * per_sm;
        h->tile_waves = (int)std::max(1LL, (total + 512LL * h->tile_slots - 1) / (512LL * h->tile_slots));
        const long long per_wave = (long long)h->tile_waves * h->tile_slots;
        h->tile_cells = (int)std::min(1024LL, std::max(64LL, (total + per_wave - 1) / per_wave));
    }
    int st;
    if ((st = dev_alloc(h, &h->d_err, 1)) != HB_OK || (st = dev_alloc(h, &h->d_ctr, 1)) != HB_OK ||
        (st = dev_alloc(h, &h->d_bar, 2)) != HB_OK) {
        delete h;
        return st;
    }
    st = h->with_mesh([&](auto &m) { return build_device_mesh(h, meshes, n, m); });
    if (st == HB_OK && opt.layout == HB_LAYOUT_TILE) st = hb_tiles_set_smem(h);
    if (st != HB_OK) { delete h; return st; }
    *out = h;
    return HB_OK;
}

extern "C" int hb_create(const hb_mesh_desc *md, const hb_options *opt_in, hb_handle **out) {
    if (!md || !out) return hb::set_error(HB_E_INVALID, "hb_create: null argument");
    return hb_create_batch(md, 1, opt_in, out);
}

extern "C" int hb_destroy(hb_handle *h) {
    delete h;
    return HB_OK;
}

extern "C" int hb_batch_size(hb_handle *h, int32_t *n) {
    if (!h || !n) return hb::set_error(HB_E_INVALID, "null argument");
    *n = (int32_t)h->scn.size();
    return HB_OK;
}

extern "C" int hb_scenario_cells(hb_handle *h, int32_t s, int32_t *cells, int32_t *first) {
    TRY(check_scenario(h, s));
    if (cells) *cells = h->scn[s].cells;
    if (first) *first = h->scn[s].cell0;
    return HB_OK;
}

namespace {
// State in and out go through the reference-order staging buffer and the
// staging kernels, which hold each precision's conversion (SplitCodec).
template <class A>
int set_state_t(hb_handle *h, int s, hb::DevMesh<A> &m, const double *H, const double *U, const double *V,
                const double *Z, const double *W) {
    using R = typename A::real;
    const hb::Scenario &sc = h->scn[s];
    const int C = sc.cells;
    const double *src[4] = {H, U, V, Z};
    for (int k = 0; k < 4; k++)
        if (!src[k]) return hb::set_error(HB_E_INVALID, "hb_set_state: missing array");
    HB_CUDA_RET(cudaDeviceSynchronize());
    for (int k = 0; k < 4; k++)
        HB_CUDA_RET(cudaMemcpy(h->d_stage + (size_t)k * C, src[k], C * sizeof(double), cudaMemcpyHostToDevice));
    hb::stage_in_kernel<A><<<(C + 255) / 256, 256>>>(m, sc.cell0, C, sc.hm1, h->d_perm + sc.cell0, h->d_stage);
    HB_CUDA_RET(cudaGetLastError());
    if (W) {
        std::vector<R> w(C);
        for (int i = 0; i < C; i++) w[i] = (R)W[sc.perm[i]];
        HB_CUDA_RET(cudaMemcpy(m.W + sc.cell0, w.data(), C * sizeof(R), cudaMemcpyHostToDevice));
    }
    HB_CUDA_RET(cudaDeviceSynchronize());
    return HB_OK;
}
template <class A>
int get_state_t(hb_handle *h, int s, hb::DevMesh<A> &m, double *H, double *U, double *V, double *Z, double *W) {
    const hb::Scenario &sc = h->scn[s];
    const int C = sc.cells;
    double *dst[5] = {H, U, V, Z, W};
    HB_CUDA_RET(cudaDeviceSynchronize());
    hb::stage_out_kernel<A><<<(C + 255) / 256, 256>>>(m, sc.cell0, C, sc.hm1, h->d_perm + sc.cell0, h->d_stage);
    HB_CUDA_RET(cudaGetLastError());
    for (int k = 0; k < 5; k++)
        if (dst[k]) HB_CUDA_RET(cudaMemcpy(dst[k], h->d_stage + (size_t)k * C, C * sizeof(double), cudaMemcpyDeviceToHost));
    return HB_OK;
}
template <class A>
int get_flux_t(hb_handle *h, int s, hb::DevMesh<A> &m, double *F0, double *F1, double *F2, double *F3) {
    using R = typename A::real;
    const hb::Scenario &sc = h->scn[s];
    const int C = sc.cells;
    const size_t S = 4 * (size_t)C;
    std::vector<R> buf(S);
    double *dst[4] = {F0, F1, F2, F3};
    R *src[4] = {m.f0, m.f1, m.f2, m.f3};
    HB_CUDA_RET(cudaDeviceSynchronize());
    for (int k = 0; k < 4; k++) {
        if (!dst[k]) continue;
        HB_CUDA_RET(cudaMemcpy(buf.data(), src[k] + 4 * (size_t)sc.cell0, S * sizeof(R), cudaMemcpyDeviceToHost));
        for (int i = 0; i < C; i++)
            for (int j = 0; j < 4; j++) dst[k][4 * (size_t)sc.perm[i] + j] = (double)buf[4 * (size_t)i + j];
    }
    return HB_OK;
}
template <class A>
int get_klas_t(hb_handle *h, int s, hb::DevMesh<A> &m, double *klas) {
    const hb::Scenario &sc = h->scn[s];
    const int C = sc.cells;
    std::vector<uint8_t> meta(std::max(sc.nrecords, 1));
    HB_CUDA_RET(cudaDeviceSynchronize());
    HB_CUDA_RET(cudaMemcpy(meta.data(), m.rmeta + sc.rec0, sc.nrecords, cudaMemcpyDeviceToHost));
    for (int i = 0; i < C; i++)
        for (int j = 0; j < 4; j++) {
            const size_t so = 4 * (size_t)sc.perm[i] + j;
            const int ci = sc.slot_index[4 * (size_t)i + j];
            const int code = ci < 0 ? hb::CODE_ZERO : (meta[ci - sc.rec0] & hb::META_CODE);
            double k = sc.klas_orig[so];
            if (hb::klas_code(k) == hb::CODE_K7 && code == hb::CODE_ZERO) k = 0.0;   // breached (functors.cu:242)
            klas[so] = k;
        }
    return HB_OK;
}
}  // namespace

extern "C" int hb_set_state_at(hb_handle *h, int32_t s, const double *H, const double *U, const double *V,
                               const double *Z, const double *W) {
    TRY(check_scenario(h, s));
    return h->with_mesh([&](auto &m) { return set_state_t(h, s, m, H, U, V, Z, W); });
}
extern "C" int hb_get_state_at(hb_handle *h, int32_t s, double *H, double *U, double *V, double *Z, double *W) {
    TRY(check_scenario(h, s));
    return h->with_mesh([&](auto &m) { return get_state_t(h, s, m, H, U, V, Z, W); });
}
extern "C" int hb_get_flux_at(hb_handle *h, int32_t s, double *F0, double *F1, double *F2, double *F3) {
    TRY(check_scenario(h, s));
    return h->with_mesh([&](auto &m) { return get_flux_t(h, s, m, F0, F1, F2, F3); });
}
extern "C" int hb_get_klas_at(hb_handle *h, int32_t s, double *klas) {
    TRY(check_scenario(h, s));
    if (!klas) return hb::set_error(HB_E_INVALID, "null argument");
    return h->with_mesh([&](auto &m) { return get_klas_t(h, s, m, klas); });
}
extern "C" int hb_set_state(hb_handle *h, const double *H, const double *U, const double *V, const double *Z, const double *W) {
    return hb_set_state_at(h, 0, H, U, V, Z, W);
}
extern "C" int hb_get_state(hb_handle *h, double *H, double *U, double *V, double *Z, double *W) {
    return hb_get_state_at(h, 0, H, U, V, Z, W);
}
extern "C" int hb_get_flux(hb_handle *h, double *F0, double *F1, double *F2, double *F3) {
    return hb_get_flux_at(h, 0, F0, F1, F2, F3);
}
extern "C" int hb_get_klas(hb_handle *h, double *klas) {
    return hb_get_klas_at(h, 0, klas);
}

extern "C" int hb_step(hb_handle *h, int32_t nsteps, void *stream) {
    NvtxRange nvtx_("hb_step");
    if (!h || nsteps < 0) return hb::set_error(HB_E_INVALID, "hb_step: bad argument");
    TRY(check_range(h, nsteps));
    TRY(enqueue_steps(h, nsteps, (cudaStream_t)stream));
    h->steps_done += nsteps;
    return HB_OK;
}

namespace {
template <class A>
int step_host_t(hb_handle *h, hb::DevMesh<A> &m, double *H, double *U, double *V, double *Z, double *W, int n,
                cudaStream_t st) {
    const hb::Scenario &sc = h->scn[0];
    const int C = sc.cells;
    const size_t b = (size_t)C * sizeof(double);
    double *io[5] = {H, U, V, Z, W};
    // arrays that follow one another in host memory (H, U, V, Z, W rows of one
    // [5][CELL] block) move as one copy, like the staging rows on the device
    auto copies = [&](int nk, cudaMemcpyKind kind) -> int {
        for (int k = 0; k < nk;) {
            if (!io[k]) { k++; continue; }
            int e = k + 1;
            while (e < nk && io[e] == io[e - 1] + C) e++;
            double *dev = h->d_stage + (size_t)k * C;
            if (kind == cudaMemcpyHostToDevice) HB_CUDA_RET(cudaMemcpyAsync(dev, io[k], b * (e - k), kind, st));
            else HB_CUDA_RET(cudaMemcpyAsync(io[k], dev, b * (e - k), kind, st));
            k = e;
        }
        return HB_OK;
    };
    TRY(copies(4, cudaMemcpyHostToDevice));
    const int blocks = (C + 255) / 256;
    hb::stage_in_kernel<A><<<blocks, 256, 0, st>>>(m, 0, C, sc.hm1, h->d_perm, h->d_stage);
    HB_CUDA_RET(cudaGetLastError());
    TRY(enqueue_steps(h, n, st));
    hb::stage_out_kernel<A><<<blocks, 256, 0, st>>>(m, 0, C, sc.hm1, h->d_perm, h->d_stage);
    HB_CUDA_RET(cudaGetLastError());
    TRY(copies(5, cudaMemcpyDeviceToHost));
    return HB_OK;
}
}  // namespace

extern "C" int hb_step_host(hb_handle *h, double *H, double *U, double *V, double *Z, double *W, int32_t nsteps,
                            void *stream) {
    NvtxRange nvtx_("hb_step_host");
    if (!h || !H || !U || !V || !Z || nsteps < 0) return hb::set_error(HB_E_INVALID, "hb_step_host: bad argument");
    if (h->segmented()) return hb::set_error(HB_E_INVALID, "hb_step_host: not available on a batch handle");
    TRY(check_range(h, nsteps));
    cudaStream_t st = (cudaStream_t)stream;
    int r = h->with_mesh([&](auto &m) { return step_host_t(h, m, H, U, V, Z, W, nsteps, st); });
    if (r == HB_OK) h->steps_done += nsteps;
    return r;
}

extern "C" int hb_sync(hb_handle *h, void *stream) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    HB_CUDA_RET(cudaStreamSynchronize((cudaStream_t)stream));
    uint32_t bits = 0;
    HB_CUDA_RET(cudaMemcpy(&bits, h->d_err, sizeof bits, cudaMemcpyDeviceToHost));
    if (bits & hb::ERRBIT_BARRIER) return hb::set_error(HB_E_BARRIER_TIMEOUT, "a grid barrier of the persistent kernel gave up waiting");
    if (bits & hb::ERRBIT_NONFINITE) return hb::set_error(HB_E_NONFINITE, "a step produced a non-finite state");
    if (bits & hb::ERRBIT_UNDEFINED) return hb::set_error(HB_E_UNDEFINED_REF, "a slot without neighbour reached the mirrored Osher branch");
    if (bits & hb::ERRBIT_TABLE_RANGE) return hb::set_error(HB_E_INVALID, "a step ran beyond the boundary tables");
    return HB_OK;
}

extern "C" int hb_set_barrier_limit(hb_handle *h, int64_t timeout_ns, int32_t phantom_arrivals) {
    if (!h || timeout_ns <= 0 || timeout_ns > 10000000000ll || phantom_arrivals < 0 || phantom_arrivals > (1 << 20))
        return hb::set_error(HB_E_INVALID, "hb_set_barrier_limit: bad argument");
    if ((unsigned long long)timeout_ns != h->barrier_limit_ns || (unsigned)phantom_arrivals != h->barrier_phantom)
        h->drop_graph();   // both are launch arguments captured by a graph
    h->barrier_limit_ns = (unsigned long long)timeout_ns;
    h->barrier_phantom = (unsigned)phantom_arrivals;
    return HB_OK;
}

extern "C" int hb_device_errors(hb_handle *h, uint32_t *bits) {
    if (!h || !bits) return hb::set_error(HB_E_INVALID, "null argument");
    HB_CUDA_RET(cudaMemcpy(bits, h->d_err, sizeof *bits, cudaMemcpyDeviceToHost));
    return HB_OK;
}

extern "C" int hb_position(hb_handle *h, int64_t *steps_done, int32_t *kt, int32_t *jt) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    const int per_day = h->scn[0].per_day;
    if (steps_done) *steps_done = h->steps_done;
    if (kt) *kt = 1 + (int)(h->steps_done % per_day);
    if (jt) *jt = (int)(h->steps_done / per_day);
    return HB_OK;
}

extern "C" int hb_set_position(hb_handle *h, int64_t steps_done) {
    if (!h || steps_done < 0) return hb::set_error(HB_E_INVALID, "hb_set_position: bad argument");
    HB_CUDA_RET(cudaDeviceSynchronize());
    // keep the state in place: it sits in buffer (steps_done & 1)
    if ((steps_done & 1) != (h->steps_done & 1)) {
        const int from = (int)(h->steps_done & 1), to = from ^ 1;
        TRY(h->with_mesh([&](auto &m) -> int {
            HB_CUDA_RET(cudaMemcpy(m.S[to], m.S[from], 4 * (size_t)h->C * sizeof(*m.S[0]), cudaMemcpyDeviceToDevice));
            return HB_OK;
        }));
    }
    long long v = steps_done;
    HB_CUDA_RET(cudaMemcpy(h->d_ctr, &v, sizeof v, cudaMemcpyHostToDevice));
    h->steps_done = steps_done;
    return HB_OK;
}

extern "C" int hb_capture_graph(hb_handle *h, int32_t nsteps, void *stream) {
    NvtxRange nvtx_("hb_capture_graph");
    if (!h || nsteps <= 0) return hb::set_error(HB_E_INVALID, "hb_capture_graph: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    cudaStream_t cap = st;
    bool own = false;
    if (!st) { HB_CUDA_RET(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)); own = true; }
    h->drop_graph();
    HB_CUDA_RET(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int st2 = enqueue_steps(h, nsteps, cap);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(cap, &g);
    if (own) cudaStreamDestroy(cap);
    if (st2 != HB_OK) { if (g) cudaGraphDestroy(g); return st2; }
    if (e != cudaSuccess) return hb::set_error(HB_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    h->graph = g;
    HB_CUDA_RET(cudaGraphInstantiate(&h->graph_exec, g, 0));
    h->graph_steps = nsteps;
    return HB_OK;
}

extern "C" int hb_graph_launch(hb_handle *h, void *stream) {
    NvtxRange nvtx_("hb_graph_launch");
    if (!h || !h->graph_exec) return hb::set_error(HB_E_INVALID, "hb_graph_launch: no graph captured");
    TRY(check_range(h, h->graph_steps));
    HB_CUDA_RET(cudaGraphLaunch(h->graph_exec, (cudaStream_t)stream));
    h->steps_done += h->graph_steps;
    return HB_OK;
}

extern "C" int hb_device_state(hb_handle *h, void **H, void **U, void **V, void **Z, void **W, int32_t *stride) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    const int par = (int)(h->steps_done & 1);
    h->with_mesh([&](auto &m) {
        auto *b = m.S[par];
        if (H) *H = b;
        if (U) *U = b + 1;
        if (V) *V = b + 2;
        // split precision keeps no level: its fourth entry is the depth's low part
        if (Z) *Z = h->opt.precision == HB_SPLIT ? nullptr : (void *)(b + 3);
        if (W) *W = m.W;
        return HB_OK;
    });
    if (stride) *stride = 4;
    return HB_OK;
}

extern "C" int hb_get_permutation(hb_handle *h, int32_t *perm) {
    return hb_get_permutation_at(h, 0, perm);
}

extern "C" int hb_get_permutation_at(hb_handle *h, int32_t s, int32_t *perm) {
    TRY(check_scenario(h, s));
    if (!perm) return hb::set_error(HB_E_INVALID, "null argument");
    memcpy(perm, h->scn[s].perm.data(), h->scn[s].perm.size() * sizeof(int32_t));
    return HB_OK;
}

extern "C" int hb_set_tile_config(hb_handle *h, int32_t tile_config) {
    if (!h) return hb::set_error(HB_E_INVALID, "null handle");
    const int c = config_for(h->opt.layout, tile_config);
    if (c < 0) return hb::set_error(HB_E_INVALID, "tile_config %d is no shape of this handle's layout", tile_config);
    if (h->opt.persistent && c != hb::DEFAULT_EDGE_CONFIG)
        return hb::set_error(HB_E_INVALID, "a persistent handle keeps the default launch shape");
    if (c != h->launch_config) h->drop_graph();
    h->launch_config = c;
    return HB_OK;
}

extern "C" int hb_get_tile_config(hb_handle *h, int32_t *tile_config) {
    if (!h || !tile_config) return hb::set_error(HB_E_INVALID, "null argument");
    *tile_config = h->launch_config + 1;
    return HB_OK;
}

// The autotuner: every launch shape runs `steps` steps from the current state
// (after one untimed step), timed with CUDA events on `stream`; the state,
// fluxes, boundary codes, error bits and step counter are restored after each
// trial and at the end, so the handle continues as if nothing had run.  The
// fastest shape becomes the handle's (a captured graph is dropped).
extern "C" int hb_autotune(hb_handle *h, int32_t steps, void *stream, float *ms_per_step, int32_t capacity,
                           int32_t *best) {
    NvtxRange nvtx_("hb_autotune");
    if (!h || steps <= 0) return hb::set_error(HB_E_INVALID, "hb_autotune: bad argument");
    if (h->opt.persistent) return hb::set_error(HB_E_INVALID, "hb_autotune: a persistent handle has one launch shape");
    TRY(check_range(h, (long long)steps + 1));
    cudaStream_t st = (cudaStream_t)stream;
    HB_CUDA_RET(cudaDeviceSynchronize());
    // snapshot of everything a step writes
    struct Piece { void *p; size_t bytes; };
    std::vector<Piece> pieces;
    h->with_mesh([&](auto &m) {
        using R = typename std::remove_reference<decltype(m)>::type::R;
        const size_t C = (size_t)h->C;
        pieces = {{m.S[0], 4 * C * sizeof(R)}, {m.S[1], 4 * C * sizeof(R)}, {m.W, C * sizeof(R)},
                  {m.f0, 4 * C * sizeof(R)}, {m.f1, 4 * C * sizeof(R)}, {m.f2, 4 * C * sizeof(R)},
                  {m.f3, 4 * C * sizeof(R)}, {m.rmeta, (size_t)std::max(m.nrecords, 1)},
                  {h->d_err, sizeof(uint32_t)}, {h->d_ctr, sizeof(long long)}};
        return HB_OK;
    });
    size_t total = 0;
    for (auto &p : pieces) total += (p.bytes + 255) & ~(size_t)255;
    char *snap = nullptr;
    {
        cudaError_t e = cudaMalloc(&snap, total);
        if (e != cudaSuccess) return hb::set_error(HB_E_NOMEM, "hb_autotune: cudaMalloc(%zu): %s", total, cudaGetErrorString(e));
    }
    auto copy_all = [&](bool save) -> int {
        size_t off = 0;
        for (auto &p : pieces) {
            if (save) HB_CUDA_RET(cudaMemcpyAsync(snap + off, p.p, p.bytes, cudaMemcpyDeviceToDevice, st));
            else HB_CUDA_RET(cudaMemcpyAsync(p.p, snap + off, p.bytes, cudaMemcpyDeviceToDevice, st));
            off += (p.bytes + 255) & ~(size_t)255;
        }
        return HB_OK;
    };
    const int saved_config = h->launch_config;
    int rc = copy_all(true);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == HB_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = hb::set_error(HB_E_CUDA, "hb_autotune: cudaEventCreate failed");
    int best_c = saved_config;
    float best_ms = 0.f;
    bool first = true;
    for (int c = 0; rc == HB_OK && c < hb::N_LAUNCH_CONFIGS; c++) {
        if (ms_per_step && c < capacity) ms_per_step[c] = 0.f;
        if (hb::LAUNCH_CONFIGS[c].layout != h->opt.layout) continue;
        h->launch_config = c;
        if ((rc = copy_all(false)) != HB_OK) break;
        if ((rc = enqueue_steps(h, 1, st)) != HB_OK) break;
        if (cudaEventRecord(e0, st) != cudaSuccess) { rc = hb::set_error(HB_E_CUDA, "cudaEventRecord"); break; }
        if ((rc = enqueue_steps(h, steps, st)) != HB_OK) break;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
            rc = hb::set_error(HB_E_CUDA, "hb_autotune: event wait failed");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)steps;
        if (ms_per_step && c < capacity) ms_per_step[c] = ms;
        if (first || ms < best_ms) { best_ms = ms; best_c = c; first = false; }
    }
    if (rc == HB_OK) rc = copy_all(false);
    cudaStreamSynchronize(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(snap);
    if (rc != HB_OK) { h->launch_config = saved_config; return rc; }
    if (best_c != saved_config) h->drop_graph();
    h->launch_config = best_c;
    if (best) *best = best_c + 1;
    return HB_OK;
}

// The reference driver's --dump file (cuda_native_impl/benchmark.cu:141-162):
// int32 CELL; H, U, V, Z [CELL]; SLCOS, SLSIN, SIDE [4*CELL]; FLUX0..3
// [4*CELL]; every value of the build's Real type (double for HB_FP64 and
// HB_SPLIT, float for HB_FP32), reference order.  The geometry comes from the
// caller's mesh description (the arrays the reference reads back from its
// host mesh); the state and fluxes from scenario s of the handle.
extern "C" int hb_write_dump(hb_handle *h, int32_t s, const hb_mesh_desc *md, const char *path) {
    TRY(check_scenario(h, s));
    if (!md || !path || !md->slcos || !md->slsin || !md->side)
        return hb::set_error(HB_E_INVALID, "hb_write_dump: null argument");
    const int C = h->scn[s].cells;
    if (md->cells != C) return hb::set_error(HB_E_INVALID, "hb_write_dump: mesh has %d cells, scenario %d", md->cells, C);
    const size_t S = 4 * (size_t)C;
    std::vector<double> st(5 * (size_t)C), fl(4 * S);
    TRY(hb_get_state_at(h, s, st.data(), st.data() + C, st.data() + 2 * (size_t)C, st.data() + 3 * (size_t)C, nullptr));
    TRY(hb_get_flux_at(h, s, fl.data(), fl.data() + S, fl.data() + 2 * S, fl.data() + 3 * S));
    FILE *f = fopen(path, "wb");
    if (!f) return hb::set_error(HB_E_IO, "hb_write_dump: cannot open %s", path);
    const bool f32 = h->opt.precision == HB_FP32;
    bool ok = fwrite(&C, sizeof(int32_t), 1, f) == 1;
    auto put = [&](const double *a, size_t n) {
        if (!ok) return;
        if (f32) {
            std::vector<float> b(a, a + n);
            ok = fwrite(b.data(), sizeof(float), n, f) == n;
        } else {
            ok = fwrite(a, sizeof(double), n, f) == n;
        }
    };
    for (int k = 0; k < 4; k++) put(st.data() + (size_t)k * C, C);
    put(md->slcos, S);
    put(md->slsin, S);
    put(md->side, S);
    for (int k = 0; k < 4; k++) put(fl.data() + (size_t)k * S, S);
    if (fclose(f) != 0) ok = false;
    return ok ? HB_OK : hb::set_error(HB_E_IO, "hb_write_dump: write to %s failed", path);
}

// ---------------------------------------------------------------------------
// checkpoint / resume
// ---------------------------------------------------------------------------
namespace {
struct CheckpointHeader {
    char magic[8];                      // "HBCKPT1"
    int32_t precision, variant, layout, tile_cells, renumber;
    int32_t cells, nrecords, nscen;
    int64_t steps_done;
    uint64_t payload;                   // bytes after the header
};

// the pieces of device memory a resumed run needs, in checkpoint order
template <class A>
std::vector<std::pair<void *, size_t>> checkpoint_pieces(hb_handle *h, hb::DevMesh<A> &m) {
    using R = typename A::real;
    const size_t C = (size_t)h->C;
    const int par = (int)(h->steps_done & 1);
    return {{m.S[par], 4 * C * sizeof(R)}, {m.W, C * sizeof(R)},       {m.f0, 4 * C * sizeof(R)},
            {m.f1, 4 * C * sizeof(R)},     {m.f2, 4 * C * sizeof(R)}, {m.f3, 4 * C * sizeof(R)},
            {m.rmeta, (size_t)m.nrecords}, {h->d_err, sizeof(uint32_t)}};
}
}  // namespace

extern "C" int hb_checkpoint_size(hb_handle *h, size_t *bytes) {
    if (!h || !bytes) return hb::set_error(HB_E_INVALID, "null argument");
    size_t n = sizeof(CheckpointHeader);
    h->with_mesh([&](auto &m) {
        for (auto &p : checkpoint_pieces(h, m)) n += p.second;
        return HB_OK;
    });
    *bytes = n;
    return HB_OK;
}

extern "C" int hb_checkpoint_save(hb_handle *h, void *buffer, size_t bytes) {
    size_t need = 0;
    TRY(hb_checkpoint_size(h, &need));
    if (!buffer || bytes < need) return hb::set_error(HB_E_INVALID, "hb_checkpoint_save: buffer of %zu bytes, need %zu", bytes, need);
    HB_CUDA_RET(cudaDeviceSynchronize());
    CheckpointHeader hd{};
    memcpy(hd.magic, "HBCKPT1", 8);
    hd.precision = h->opt.precision; hd.variant = h->opt.variant; hd.layout = h->opt.layout;
    hd.tile_cells = h->opt.tile_cells; hd.renumber = h->opt.renumber;
    hd.cells = h->C; hd.nscen = (int32_t)h->scn.size();
    hd.steps_done = h->steps_done;
    hd.payload = need - sizeof hd;
    char *out = (char *)buffer + sizeof hd;
    int rc = h->with_mesh([&](auto &m) -> int {
        hd.nrecords = m.nrecords;
        for (auto &p : checkpoint_pieces(h, m)) {
            HB_CUDA_RET(cudaMemcpy(out, p.first, p.second, cudaMemcpyDeviceToHost));
            out += p.second;
        }
        return HB_OK;
    });
    if (rc != HB_OK) return rc;
    memcpy(buffer, &hd, sizeof hd);
    return HB_OK;
}

extern "C" int hb_checkpoint_load(hb_handle *h, const void *buffer, size_t bytes) {
    if (!h || !buffer || bytes < sizeof(CheckpointHeader)) return hb::set_error(HB_E_INVALID, "hb_checkpoint_load: bad argument");
    CheckpointHeader hd;
    memcpy(&hd, buffer, sizeof hd);
    if (memcmp(hd.magic, "HBCKPT1", 8) != 0) return hb::set_error(HB_E_INVALID, "hb_checkpoint_load: not a checkpoint");
    int nrec = 0;
    h->with_mesh([&](auto &m) { nrec = m.nrecords; return HB_OK; });
    if (hd.precision != h->opt.precision || hd.variant != h->opt.variant || hd.layout != h->opt.layout ||
        hd.tile_cells != h->opt.tile_cells || hd.renumber != h->opt.renumber || hd.cells != h->C ||
        hd.nscen != (int32_t)h->scn.size() || hd.nrecords != nrec)
        return hb::set_error(HB_E_INVALID, "hb_checkpoint_load: the checkpoint is of another mesh or other options");
    if (hd.steps_done < 0 || hd.steps_done > h->step_limit())
        return hb::set_error(HB_E_INVALID, "hb_checkpoint_load: position %lld beyond the boundary tables", (long long)hd.steps_done);
    if (bytes < sizeof hd + hd.payload) return hb::set_error(HB_E_INVALID, "hb_checkpoint_load: truncated checkpoint");
    HB_CUDA_RET(cudaDeviceSynchronize());
    h->steps_done = hd.steps_done;   // the state goes into buffer (steps_done & 1)
    const char *in = (const char *)buffer + sizeof hd;
    int rc = h->with_mesh([&](auto &m) -> int {
        for (auto &p : checkpoint_pieces(h, m)) {
            HB_CUDA_RET(cudaMemcpy(p.first, in, p.second, cudaMemcpyHostToDevice));
            in += p.second;
        }
        return HB_OK;
    });
    if (rc != HB_OK) return rc;
    long long v = hd.steps_done;
    HB_CUDA_RET(cudaMemcpy(h->d_ctr, &v, sizeof v, cudaMemcpyHostToDevice));
    return HB_OK;
}


// ---------------------------------------------------------------------------
// halo exchange of a mesh split across handles
// ---------------------------------------------------------------------------
namespace {

// buf[i] = the state record of cell cells[i] (pack) or the reverse (unpack);
// a record is the four state components of one cell.
template <class R>
__global__ void halo_pack_kernel(const R *__restrict__ S, const int32_t *__restrict__ cells, int n,
                                 R *__restrict__ buf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const hb::Vec4<R> v = hb::ld4(S + 4 * (size_t)cells[i]);
    hb::st4(buf + 4 * (size_t)i, v.x, v.y, v.z, v.w);
}
template <class R>
__global__ void halo_unpack_kernel(R *__restrict__ S, const int32_t *__restrict__ cells, int n,
                                   const R *__restrict__ buf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const hb::Vec4<R> v = hb::ld4(buf + 4 * (size_t)i);
    hb::st4(S + 4 * (size_t)cells[i], v.x, v.y, v.z, v.w);
}

int halo_args(hb_handle *h, int32_t list, const void *buf, const char *who) {
    if (!h || !buf) return hb::set_error(HB_E_INVALID, "%s: null argument", who);
    if (list < 0 || list >= (int32_t)h->halo_lists.size())
        return hb::set_error(HB_E_INVALID, "%s: no halo list %d", who, list);
    if ((uintptr_t)buf % 16 != 0) return hb::set_error(HB_E_INVALID, "%s: buffer not 16-byte aligned", who);
    return HB_OK;
}

}  // namespace

extern "C" int hb_state_record_bytes(const hb_handle *h, int32_t *bytes) {
    if (!h || !bytes) return hb::set_error(HB_E_INVALID, "null argument");
    *bytes = h->opt.precision == HB_FP64 ? 32 : 16;
    return HB_OK;
}

extern "C" int hb_halo_define(hb_handle *h, const int32_t *cells, int32_t n, int32_t *list) {
    if (!h || !list || n < 0 || (n > 0 && !cells)) return hb::set_error(HB_E_INVALID, "hb_halo_define: bad argument");
    if (h->segmented()) return hb::set_error(HB_E_INVALID, "hb_halo_define: a batch handle has no single mesh to split");
    const hb::Scenario &sc = h->scn[0];
    std::vector<int32_t> dev(std::max(n, 1), 0);
    for (int32_t i = 0; i < n; i++) {
        if (cells[i] < 0 || cells[i] >= sc.cells)
            return hb::set_error(HB_E_INVALID, "hb_halo_define: cell %d outside 0..%d", cells[i], sc.cells - 1);
        dev[i] = sc.cell0 + sc.inv[cells[i]];
    }
    int32_t *d = nullptr;
    TRY(dev_upload(h, &d, dev));
    h->halo_lists.push_back({d, n});
    *list = (int32_t)h->halo_lists.size() - 1;
    return HB_OK;
}

extern "C" int hb_halo_pack(hb_handle *h, int32_t list, void *buf, void *stream) {
    TRY(halo_args(h, list, buf, "hb_halo_pack"));
    const auto L = h->halo_lists[list];
    if (L.n == 0) return HB_OK;
    const int par = (int)(h->steps_done & 1);
    return h->with_mesh([&](auto &m) -> int {
        using R = std::remove_pointer_t<std::decay_t<decltype(m.S[0])>>;
        halo_pack_kernel<R><<<(L.n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(m.S[par], L.cells, L.n, (R *)buf);
        HB_CUDA_RET(cudaGetLastError());
        return HB_OK;
    });
}

extern "C" int hb_halo_unpack(hb_handle *h, int32_t list, const void *buf, void *stream) {
    TRY(halo_args(h, list, buf, "hb_halo_unpack"));
    const auto L = h->halo_lists[list];
    if (L.n == 0) return HB_OK;
    const int par = (int)(h->steps_done & 1);
    return h->with_mesh([&](auto &m) -> int {
        using R = std::remove_pointer_t<std::decay_t<decltype(m.S[0])>>;
        halo_unpack_kernel<R><<<(L.n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(m.S[par], L.cells, L.n,
                                                                                     (const R *)buf);
        HB_CUDA_RET(cudaGetLastError());
        return HB_OK;
    });
}
