// hb_adjoint.cu -- reverse-mode adjoint of the fp64 timestep (variant H).
//
// A rollout of T steps x_{t+1} = F(x_t; n, ZBC) from the initial level and
// velocities, with the loss
//     L = sum over observation steps t (every `obs_every`) and gauge cells g
//         of (H_t[g] - Hobs_t[g])^2,
// and its gradient with respect to the per-cell Manning coefficient n
// (FNC = 9.81 n^2, mesh.cpp:364) and bed elevation ZBC.  The initial depth
// follows the bed as in mesh.cpp:350-361: H0 = Z0 - ZBC where Z0 > ZBC, else
// H0 = HM1 and Z0 = ZBC + HM1.
//
// The reverse sweep is written out by hand.  Every branch choice of the
// forward step (the slot's branch chain and Osher's wave case, wet/dry and
// velocity clamps, max/min picks, the iteration counts of the KLAS 10 and
// KLAS 1 fixed points) is taken from the forward state, recomputed with the
// forward's own arithmetic, and the derivative is that of the chosen branch.
// Adjoint arithmetic is plain fp64.
//
// Memory: the state is kept every `checkpoint_every` = k steps; the backward
// pass recomputes each k-step segment from its checkpoint, keeping that
// segment's states and the update coefficients of its steps (written by
// the recomputed update kernels), then runs the segment's reverse steps, one
// kernel each (adj_step_kernel, four lanes per cell):
//   - the state adjoint after the step, gathered from the later step's
//     direct terms, the cell's own slots' contributions and those of the
//     neighbours' slots that face it (fixed order, no atomics: the gradient
//     is deterministic);
//   - lane 0: the cell update's reverse (from the stored coefficients),
//     shared with the other lanes;
//   - lane j: slot j's flux reverse, leaving its contributions to its own
//     cell and its neighbour for the next (earlier) step.
// The forward rollout is replayed from a CUDA graph of k steps whose
// checkpoint and gauge kernels take their slot from the device step counter.
#include <cmath>
#include <cstring>
#include <vector>

#include "hb_handle.hpp"

namespace hb {
namespace adj {

using A = F64Exact;

// adjoint of one cell's slot inputs {h, u, v, z, zbc}
struct Adj5 { double h, u, v, z, b; };

// A slot's Adj5 contribution in memory: six doubles (the last one padding),
// moved as three aligned 16-byte accesses.  (Eight doubles moved as two
// 256-bit accesses measured slower: the extra bytes cost more than the
// saved instruction.)
constexpr int ADJ_REC = 6;
__device__ __forceinline__ void ld_rec(const double *p, double q[5]) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    const double2 c = reinterpret_cast<const double2 *>(p)[2];
    q[0] = a.x; q[1] = a.y; q[2] = b.x; q[3] = b.y; q[4] = c.x;
}
__device__ __forceinline__ void st_rec(double *p, const Adj5 &g) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(g.h, g.u);
    reinterpret_cast<double2 *>(p)[1] = make_double2(g.v, g.z);
    reinterpret_cast<double2 *>(p)[2] = make_double2(g.b, 0.0);
}

// QF(h, u, v) = (h u, h u^2, h u v, 4.905 h^2) times `sign`, reversed with
// output adjoint ob (functors.cu:505-511)
__device__ __forceinline__ void qf_rev(double h, double u, double v, double sign, const double ob[4], double &hb,
                                       double &ub, double &vb) {
    hb += sign * (ob[0] * u + ob[1] * u * u + ob[2] * u * v + ob[3] * 9.81 * h);
    ub += sign * (ob[0] * h + ob[1] * 2.0 * h * u + ob[2] * h * v);
    vb += sign * (ob[2] * h * u);
}

// Forward values of one Osher evaluation (functors.cu:570-712) that its
// reverse needs: the case, every piece's (h, u) and FLUX3, all computed with
// the forward's own arithmetic (osher() in hb_physics.cuh), so the case and
// FLUX3 are the forward's bit for bit.
struct OsherFwd {
    bool p1, p2, p3, p5, p6, p7;
    double s2, s6;                       // signs of pieces 2 and 6
    double cr, fir, us, hs, ua35, fil3, ha3, fir5, ha5, us6, hs6;
    double fo3;
};

__device__ __forceinline__ OsherFwd osher_fwd(double cl, const double ql[3], const double qr[3], double fil) {
    OsherFwd o;
    o.cr = A::sqrt(A::mul(A::c(9.81), qr[0]));
    o.fir = A::sub(qr[1], A::mul(A::c(2.0), o.cr));
    const double ua = A::mul(A::add(fil, o.fir), A::c(0.5));
    const double ca = A::fabs(A::mul(A::sub(fil, o.fir), A::c(0.25)));
    int k2 = 0, k1 = 0;
    if (ca < ua) k2 = 1;
    else if (ua >= 0.0 && ua < ca) k2 = 2;
    else if (ua >= -ca && ua < 0.0) k2 = 3;
    else if (ua < -ca) k2 = 4;
    if (ql[1] < cl && qr[1] >= -o.cr) k1 = 1;
    else if (ql[1] >= cl && qr[1] >= -o.cr) k1 = 2;
    else if (ql[1] < cl && qr[1] < -o.cr) k1 = 3;
    else if (ql[1] >= cl && qr[1] < -o.cr) k1 = 4;
    const bool any = k1 != 0 && k2 != 0;
    o.p1 = any && (k1 == 2 || k1 == 4);
    o.p2 = any && (k2 == 1 ? (k1 == 1 || k1 == 3) : (k1 == 2 || k1 == 4));
    o.s2 = k2 != 1 ? -1.0 : 1.0;
    o.p3 = any && k2 == 2;
    o.p5 = any && k2 == 3;
    o.p6 = any && (k2 == 4 ? k1 <= 2 : k1 >= 3);
    o.s6 = k2 != 4 ? -1.0 : 1.0;
    o.p7 = any && k1 >= 3;
    // the dividing pieces only where the case takes them (osher() does the same)
    o.ua35 = A::mul(A::add(fil, o.fir), A::c(0.5));
    o.fil3 = A::sub(fil, o.ua35);
    o.fir5 = A::sub(o.fir, o.ua35);
    o.us = o.hs = o.ha3 = o.ha5 = o.us6 = o.hs6 = 0.0;
    if (o.p2) {
        o.us = A::divk(fil, 3.0);
        o.hs = A::divk(A::mul(o.us, o.us), 9.81);
    }
    if (o.p3) o.ha3 = A::divk(A::mul(o.fil3, o.fil3), 39.24);
    if (o.p5) o.ha5 = A::divk(A::mul(o.fir5, o.fir5), 39.24);
    if (o.p6) {
        o.us6 = A::divk(o.p5 ? o.fir5 : o.fir, 3.0);
        o.hs6 = A::divk(A::mul(o.us6, o.us6), 9.81);
    }
    // FLUX3 as qf_acc_if sums it: out3 += +-4.905 h * h over the active pieces in order
    double o3 = 0.0;
    auto acc = [&](bool on, double sign, double h) {
        const double h4 = A::mul(A::c(4.905), h);
        const double v = A::madd(sign < 0 ? -h4 : h4, h, o3, M_ACC123);
        if (on) o3 = v;
    };
    acc(o.p1, 1.0, ql[0]);
    acc(o.p2, o.s2, o.hs);
    acc(o.p3, 1.0, o.ha3);
    acc(o.p5, 1.0, o.ha5);
    acc(o.p6, o.s6, o.hs6);
    acc(o.p7, 1.0, qr[0]);
    o.fo3 = o3;
    return o;
}

// Reverse of osher() for the case its forward picked.  In: the forward values
// and the adjoint fb of out[4].  Out (added): ql_b, qr_b, fil_b.  cl enters
// only the case choice.
__device__ __forceinline__ void osher_rev(const OsherFwd &o, const double ql[3], const double qr[3], const double fb[4],
                                          double qlb[3], double qrb[3], double &filb) {
    constexpr double R3 = 1.0 / 3.0, R981 = 1.0 / 9.81, R3924 = 1.0 / 39.24;
    double firb = 0.0, ua35b = 0.0, fir5b = 0.0;
    if (o.p1) qf_rev(ql[0], ql[1], ql[2], 1.0, fb, qlb[0], qlb[1], qlb[2]);
    if (o.p2) {
        double hsb = 0.0, usb = 0.0;
        qf_rev(o.hs, o.us, ql[2], o.s2, fb, hsb, usb, qlb[2]);
        usb += hsb * 2.0 * o.us * R981;
        filb += usb * R3;
    }
    if (o.p3) {
        double hab = 0.0;
        qf_rev(o.ha3, o.ua35, ql[2], 1.0, fb, hab, ua35b, qlb[2]);
        const double fil3b = hab * 2.0 * o.fil3 * R3924;
        filb += fil3b;
        ua35b -= fil3b;
    }
    if (o.p5) {
        double hab = 0.0;
        qf_rev(o.ha5, o.ua35, qr[2], 1.0, fb, hab, ua35b, qrb[2]);
        fir5b += hab * 2.0 * o.fir5 * R3924;
    }
    if (o.p6) {
        double hsb = 0.0, usb = 0.0;
        qf_rev(o.hs6, o.us6, qr[2], o.s6, fb, hsb, usb, qrb[2]);
        usb += hsb * 2.0 * o.us6 * R981;
        const double f6b = usb * R3;
        if (o.p5) fir5b += f6b;
        else firb += f6b;
    }
    if (o.p7) qf_rev(qr[0], qr[1], qr[2], 1.0, fb, qrb[0], qrb[1], qrb[2]);
    firb += fir5b;
    ua35b -= fir5b;
    filb += 0.5 * ua35b;
    firb += 0.5 * ua35b;
    qrb[1] += firb;
    const double crb = -2.0 * firb;
    if (o.cr > 0.0) qrb[0] += crb * 9.81 * 0.5 / o.cr;
}

// Reverse of the Osher route of a slot (functors.cu:151-200): left cell L,
// right cell R, normal (cs, sn) from L to R; `mir` = the mirrored route
// (left = the neighbour).  fb: adjoint of the slot's fluxes.
__device__ void osher_route_rev(const CellStateA<A> &L, const CellStateA<A> &R, double cs, double sn, bool mir,
                                const StepParams &p, const double fb[4], Adj5 &Lb, Adj5 &Rb) {
    const double HM1 = p.hm1, HM2 = p.hm2;
    const double clL = A::sqrt(A::mul(A::c(9.81), L.h));
    const OsherIn<double> oi = osher_inputs<A>(L, R, cs, sn, clL, mir, p);
    const OsherFwd of = osher_fwd(oi.cl, oi.ql, oi.qr, oi.fil);
    // outputs: F0 = +-fo0, F1 = fo1 + (1-ratio) hcR ur^2 / 2, F2 = fo2, F3 = fo3 or mirror_f3(fo3)
    double fob[4] = {mir ? -fb[0] : fb[0], fb[1], fb[2], 0.0};
    if (!mir) {
        fob[3] = fb[3];
    } else {
        // F3 = 4.905 hc3^2, hc3 = za - ZBC_R where za = sqrt(fo3/4.905) + ZBC_L > ZBC_R (functors.cu:191-199)
        const double za = A::ladd(A::lvl(A::sqrt(A::divk(of.fo3, 4.905))), L.zbc);
        if (za > R.zbc) {
            const double hc3 = za - R.zbc;
            const double hc3b = fb[3] * 9.81 * hc3;
            Rb.b -= hc3b;
            Lb.b += hc3b;
            const double t = sqrt(of.fo3 * (1.0 / 4.905));
            if (t > 0.0) fob[3] = hc3b * (0.5 / 4.905) / t;
        }
    }
    double ratiob = 0.0, hcRb = 0.0, urb = 0.0;
    ratiob -= fb[1] * oi.hcR * oi.ur * oi.ur * 0.5;
    hcRb += fb[1] * (1.0 - oi.ratio) * oi.ur * oi.ur * 0.5;
    urb += fb[1] * (1.0 - oi.ratio) * oi.hcR * oi.ur;
    double qlb[3] = {0, 0, 0}, qrb[3] = {0, 0, 0}, filb = 0.0;
    osher_rev(of, oi.ql, oi.qr, fob, qlb, qrb, filb);
    // fil = ql1 + 2 clL, clL = sqrt(9.81 h_L)
    qlb[1] += filb;
    if (clL > 0.0) Lb.h += filb * 9.81 / clL;
    // ql = (h_L, u_L cs + v_L sn, v_L cs - u_L sn)
    Lb.h += qlb[0];
    Lb.u += qlb[1] * cs - qlb[2] * sn;
    Lb.v += qlb[1] * sn + qlb[2] * cs;
    // qr2 = v_R cs - u_R sn
    Rb.v += qrb[2] * cs;
    Rb.u -= qrb[2] * sn;
    // qr1 = ur * ratio unless clamped to +-VMIN
    if (!(oi.hcR <= HM2 || oi.qr[0] <= HM2)) {
        urb += qrb[1] * oi.ratio;
        ratiob += qrb[1] * oi.ur;
    }
    double qr0b = qrb[0];
    // ratio = min(hcR / qr0, 1.5)
    const double q = A::div(oi.hcR, oi.qr[0]);
    if (q < 1.5) {
        hcRb += ratiob / oi.qr[0];
        qr0b -= ratiob * oi.hcR / (oi.qr[0] * oi.qr[0]);
    }
    // ur = u_R cs + v_R sn
    Rb.u += urb * cs;
    Rb.v += urb * sn;
    // qr0 = max(zR - ZBC_L, HM1), zR = max(ZBC_R, Z_R)
    const double zR = A::lmax(R.zbc, R.z);
    if (A::depth(zR, L.zbc) > HM1) {
        if (R.z > R.zbc) Rb.z += qr0b;
        else Rb.b += qr0b;
        Lb.b -= qr0b;
    }
    // hcR = max(h_R, HM1)
    if (R.h > HM1) Rb.h += hcRb;
}

// Reverse of the boundary slots of BOUNDA (functors.cu:513-568) for KLAS 4,
// 10 and 1 (variant H).  hb/ql1b/ql2b/filb: adjoints of the slot's own depth,
// rotated velocity and FIL; b1b that of its bed.
template <class TableFetch>
__device__ void bounda_rev(const SlotInA<A> &in, const StepParams &p, double ql1, double ql2, double fil, double cl,
                           const TableFetch &fetch, const double fb[4], double &hb, double &ql1b, double &ql2b,
                           double &filb, double &b1b, uint32_t *err) {
    const double h = in.own.h;
    const double HM2 = p.hm2;
    const bool super = ql1 > cl && h < HM2;   // variant H (functors.cu:517)
    if (super) {
        hb += fb[0] * ql1 + fb[1] * ql1 * ql1 + fb[2] * ql1 * ql2 + fb[3] * 9.81 * h;
        ql1b += fb[0] * h + fb[1] * 2.0 * h * ql1 + fb[2] * h * ql2;
        ql2b += fb[2] * h * ql1;
        return;
    }
    switch (in.code) {
    case CODE_K4:
        hb += fb[3] * 9.81 * h;
        break;
    case CODE_K10: {   // functors.cu:204-232
        BoundaryInA<A> b = fetch();
        double f0 = -A::madd(b.dqt, A::c((double)p.kt), b.qt, M_K10);
        f0 = A::div(f0, in.side);
        // forward iterates of inflow_depth
        double hb0s[21];
        hb0s[0] = h;
        double hbv = 0.0;
        int K = 0;
        for (int k = 1; k <= 20; k++) {
            const double w = A::sub(fil, A::div(f0, hb0s[k - 1]));
            hbv = A::divk(A::mul(w, w), 39.24);
            K = k;
            if (A::fabs(A::sub(hb0s[k - 1], hbv)) <= A::c(0.005)) break;
            hb0s[k] = A::add(A::mul(hb0s[k - 1], A::c(0.5)), A::mul(hbv, A::c(0.5)));
        }
        // F1 = hb <= 1 ? 0 : f0^2 / hb, F3 = 4.905 hb^2
        double hbb = fb[3] * 9.81 * hbv;
        if (!(hbv <= 1.0)) hbb -= fb[1] * f0 * f0 / (hbv * hbv);
        // back through the iterations: hb_k = (fil - f0/hb0_{k-1})^2 / 39.24,
        // hb0_k = (hb0_{k-1} + hb_k) / 2
        double hb_k_b = hbb;      // adjoint of hb_k for the current k
        double hb0_b = 0.0;       // adjoint of hb0_{k-1} through hb0_k's average
        for (int k = K; k >= 1; k--) {
            const double w = fil - f0 / hb0s[k - 1];
            const double wb = hb_k_b * 2.0 * w / 39.24;
            filb += wb;
            const double hb0prev_b = wb * f0 / (hb0s[k - 1] * hb0s[k - 1]) + hb0_b;
            if (k - 1 >= 1) {
                hb_k_b = 0.5 * hb0prev_b;
                hb0_b = 0.5 * hb0prev_b;
            } else {
                hb += hb0prev_b;   // hb0_0 = h
            }
        }
        break;
    }
    case CODE_K1: {   // functors.cu:371-392, variant H: DZT * jt
        BoundaryInA<A> b = fetch();
        const double lev = A::lmadd(b.dzt, A::lc((double)p.jt), b.zt, M_K1);
        const double d = A::lsub(lev, in.own.zbc);
        const double hb1 = A::fmax(d, A::c(p.hm2));
        // forward iterates of invariant_iter
        const double fial = A::madd(A::c(6.264), A::sqrt(h), ql1, M_FIAL1);
        const double shb = A::sqrt(hb1);
        double us[31];
        us[0] = ql1;
        double ur0 = ql1, urb = ql1;
        int K = 0;
        for (int k = 1; k <= 30; k++) {
            const double fiar = A::madd(A::c(-6.264), shb, urb, M_FIAR1);
            const double dsum = A::add(fial, fiar), ddif = A::sub(fial, fiar);
            urb = A::divk(A::div(A::mul(A::mul(dsum, ddif), ddif), hb1), 313.92);
            us[k] = urb;
            K = k;
            if (A::fabs(A::sub(urb, ur0)) <= A::c(0.0001)) break;
            ur0 = urb;
        }
        // F0 = hb1 urb, F1 = hb1 urb^2, F3 = 4.905 hb1^2; F2 from the prelude
        double ub = fb[0] * hb1 + fb[1] * 2.0 * hb1 * urb;
        double hb1b = fb[0] * urb + fb[1] * urb * urb + fb[3] * 9.81 * hb1;
        double fialb = 0.0, shbb = 0.0;
        for (int k = K; k >= 1; k--) {
            const double fiar = us[k - 1] - 6.264 * shb;
            const double dsum = fial + fiar, ddif = fial - fiar;
            const double g = us[k];
            const double dsumb = ub * ddif * ddif / (hb1 * 313.92);
            const double ddifb = ub * 2.0 * dsum * ddif / (hb1 * 313.92);
            hb1b -= ub * g / hb1;
            fialb += dsumb + ddifb;
            const double fiarb = dsumb - ddifb;
            shbb -= 6.264 * fiarb;
            ub = fiarb;          // adjoint of us[k-1]
        }
        ql1b += ub;              // us[0] = ql1
        ql1b += fialb;
        if (h > 0.0) hb += fialb * 6.264 / (2.0 * sqrt(h));
        if (shb > 0.0) hb1b += shbb / (2.0 * shb);
        if (d > p.hm2) b1b -= hb1b;
        // prelude FLUX2 = h ql1 ql2 when ql1 > 0
        if (ql1 > 0.0) {
            hb += fb[2] * ql1 * ql2;
            ql1b += fb[2] * h * ql2;
            ql2b += fb[2] * h * ql1;
        }
        break;
    }
    default:
        atomicOr(err, ERRBIT_UNDEFINED);   // rejected at creation; never reached
        break;
    }
}

// Reverse of one slot's flux (functors.cu:47-202, variant H) for fluxes'
// adjoint fb; adds the adjoints of the own cell's and the neighbour's
// {h, u, v, z, zbc}.
template <class TableFetch>
__device__ void slot_rev(const SlotInA<A> &in, const StepParams &p, const TableFetch &fetch, const double fb[4],
                         Adj5 &go, Adj5 &gn, uint32_t *err) {
    const double HM1 = p.hm1, HM2 = p.hm2, C1 = K::C1;
    const double h1 = in.own.h, u1 = in.own.u, v1 = in.own.v, z1 = in.own.z, b1 = in.own.zbc;
    const double cs = in.cosj, sn = in.sinj;
    const double ql1 = A::dot(u1, cs, v1, sn, M_QL1);
    const double ql2 = A::dot(v1, cs, -u1, sn, M_QL2);
    const double zb1 = A::ladd(b1, A::lc(p.hm1));
    const double zi = A::lmax(z1, zb1);
    double hc = 0, bc = 0, zc = 0, uc = 0, vc = 0;
    if (in.has_nb) {
        hc = A::fmax(in.nb.h, HM1);
        bc = in.nb.zbc;
        zc = A::lmax(bc, in.nb.z);
        uc = in.nb.u;
        vc = in.nb.v;
    }
    double ql1b = 0, ql2b = 0, zib = 0, hcb = 0, bcb = 0, zcb = 0, ucb = 0, vcb = 0;
    const double cl = A::sqrt(A::mul(A::c(9.81), h1));
    if (code_is_bounda(in.code)) {
        const double fil = A::add(ql1, A::mul(A::c(2.0), cl));
        double filb = 0.0;
        bounda_rev(in, p, ql1, ql2, fil, cl, fetch, fb, go.h, ql1b, ql2b, filb, go.b, err);
        ql1b += filb;
        if (cl > 0.0) go.h += 2.0 * filb * 9.81 / (2.0 * cl);
    } else if (h1 <= HM1 && hc <= HM1) {
        // all fluxes zero
    } else if (zi <= bc) {
        hcb += fb[0] * (-C1) * 1.5 * sqrt(hc);
        go.h += fb[1] * ql1 * fabs(ql1) + fb[3] * 9.81 * h1;
        ql1b += fb[1] * h1 * 2.0 * fabs(ql1);
    } else if (zc <= b1) {
        go.h += fb[0] * C1 * 1.5 * sqrt(h1) + fb[1] * ql1 * fabs(ql1) + fb[2] * fabs(ql1) * ql2;
        ql1b += fb[1] * 2.0 * h1 * fabs(ql1) + fb[2] * h1 * (ql1 > 0 ? 1.0 : ql1 < 0 ? -1.0 : 0.0) * ql2;
        ql2b += fb[2] * h1 * fabs(ql1);
    } else if (h1 <= HM2) {
        if (zc > zi) {
            const double dz = A::depth(zc, b1);
            const double dh = A::fmax(dz, HM1);
            const double sq = sqrt(dh);
            const double vt = A::dot(vc, cs, -uc, sn, M_SHALLOW_VT);
            const double F0 = -C1 * dh * sq;
            const double dhb = fb[0] * (-C1 * 1.5 * sq) + fb[1] * (C1 * C1 * 2.0 * dh) + fb[2] * vt * (-C1 * 1.5 * sq);
            const double vtb = fb[2] * F0;
            vcb += vtb * cs;
            ucb -= vtb * sn;
            go.h += fb[3] * 9.81 * h1;
            if (dz > HM1) { zcb += dhb; go.b -= dhb; }
        } else {
            go.h += fb[0] * C1 * 1.5 * sqrt(h1) + fb[3] * 9.81 * h1;
        }
    } else if (hc <= HM2) {
        if (zi > zc) {
            const double dz = A::depth(zi, bc);
            const double dh = A::fmax(dz, HM1);
            const double sq = sqrt(dh);
            const double hc1 = A::depth(zc, b1);
            const double F0 = C1 * dh * sq;
            const double dhb = fb[0] * (C1 * 1.5 * sq) + fb[1] * (C1 * C1 * 2.0 * dh) + fb[2] * ql2 * (C1 * 1.5 * sq);
            ql2b += fb[2] * F0;
            const double hc1b = fb[3] * 9.81 * hc1;
            zcb += hc1b;
            go.b -= hc1b;
            if (dz > HM1) { zib += dhb; bcb -= dhb; }
        } else {
            hcb += fb[0] * (-C1) * 1.5 * sqrt(hc);
            go.h += fb[1] * ql1 * ql1 + fb[3] * 9.81 * h1;
            ql1b += fb[1] * 2.0 * h1 * ql1;
        }
    } else if (!(in.code == CODE_ZERO && in.own_first) && !in.has_nb) {
        atomicOr(err, ERRBIT_UNDEFINED);
    } else {
        // Osher: direct from the lower-numbered side, mirrored otherwise (one call site)
        const bool mir = !(in.code == CODE_ZERO && in.own_first);
        Adj5 lb{0, 0, 0, 0, 0}, rb{0, 0, 0, 0, 0};
        osher_route_rev(mir ? in.nb : in.own, mir ? in.own : in.nb, mir ? -cs : cs, mir ? -sn : sn, mir, p, fb, lb, rb);
        Adj5 &gl = mir ? gn : go, &gr = mir ? go : gn;
        gl.h += lb.h; gl.u += lb.u; gl.v += lb.v; gl.z += lb.z; gl.b += lb.b;
        gr.h += rb.h; gr.u += rb.u; gr.v += rb.v; gr.z += rb.z; gr.b += rb.b;
    }
    // ql = (h1, u1 cs + v1 sn, v1 cs - u1 sn)
    go.u += ql1b * cs - ql2b * sn;
    go.v += ql1b * sn + ql2b * cs;
    // zi = max(z1, ZBC + HM1)
    if (z1 >= zb1) go.z += zib;
    else go.b += zib;
    if (in.has_nb) {
        if (in.nb.h > HM1) gn.h += hcb;
        gn.b += bcb;
        if (in.nb.z > bc) gn.z += zcb;
        else gn.b += zcb;
        gn.u += ucb;
        gn.v += vcb;
    }
}

// Adjoint-side mesh: per device slot its geometry, neighbour, code and the
// neighbour's slot that faces back.
struct AdjMesh {
    const double *cs4, *sn4, *side4;
    const int32_t *nbr4, *mirror4;
    const uint8_t *meta4;        // code | own_first | has_nb; 0xFF = no real slot
    const int32_t *gauge_of;     // [C] gauge index of the cell, -1
    double *fnc_g, *zbc_g;       // [C] accumulated gradients
    double *lam;                 // [C][4] state adjoint {H, U, V, Z} (the seed, and at the end that of x_0)
    const double *res;           // [nobs][ng] residuals H - Hobs
    int ng, obs_every;
};

// What one reverse step leaves for the next (earlier) one: per cell the
// update's direct terms of the state adjoint; per slot its contributions to
// its own cell and to its neighbour ({h, u, v, z, zbc} each).  Two copies,
// step t writing copy (t & 1) and reading the other.
struct AdjStepBufs {
    const double *dir_in, *so_in, *sn_in;   // step t + 1's
    double *dir_out, *so_out, *sn_out;       // step t's
};

// lambda(c) = dir(c) + sum_j so[4c+j] + sum_j sn[mirror(4c+j)] (+ the loss
// term of observation row `obs_row`) and c's bed terms, by the four lanes of
// cell c: lane j adds slot j's pair of contributions, a butterfly over the
// four lanes sums them.  Every lane of the warp must call this.
__device__ __forceinline__ void gather4(const AdjMesh &a, const double *dir, const double *so, const double *sn,
                                        int c, int j, int obs_row, double l[4], double &zg) {
    const size_t s = 4 * (size_t)c + j;
    double part[5];
    ld_rec(so + ADJ_REC * s, part);
    const int mj = a.mirror4[s];
    if (mj >= 0) {
        double q5[5];
        ld_rec(sn + ADJ_REC * (size_t)mj, q5);
        for (int q = 0; q < 5; q++) part[q] += q5[q];
    }
    for (int q = 0; q < 5; q++) {
        part[q] += __shfl_xor_sync(0xffffffffu, part[q], 1);
        part[q] += __shfl_xor_sync(0xffffffffu, part[q], 2);
    }
    const Vec4<double> d = ldg4(dir + 4 * (size_t)c);
    l[0] = d.x + part[0]; l[1] = d.y + part[1]; l[2] = d.z + part[2]; l[3] = d.w + part[3];
    zg = part[4];
    if (obs_row >= 0) {
        const int g = a.gauge_of[c];
        if (g >= 0) l[0] += 2.0 * a.res[(size_t)obs_row * a.ng + g];
    }
}

// The update coefficients of a step (update_cell with COEF, written by the
// recomputed step's update kernel) for the reverse of the cell update.
struct UpdateCoef { double dtw, ih2, d_fnc, d_h, d_s; };
__device__ __forceinline__ UpdateCoef ld_coef(const double *p) {
    const Vec4<double> a = ldg4(p), b = ldg4(p + 4);
    return {a.x, a.y, a.z, a.w, b.x};
}

// One reverse step t, four lanes per cell.  x: the state before the step; xn:
// the state after it.  The adjoint of the state after the step is gathered
// first from step t + 1's contributions (`first`: it is the seed a.lam
// instead), with the loss term of row `obs_row` when step t + 1 ends on an
// observation.  Lane 0 reverses the cell update and shares the adjoints of the
// slot sums; lane j then reverses slot j.
//
// coef: the step's update coefficients (written with the recomputed step).
//
// The update's forward values come from xn rather than from the slot sums:
// H2 = max(H + QLUA - DTA WH, HM1) is xn's depth, so H2 > HM1 exactly when the
// unclamped depth is; and where H2 > HM2 the velocity U2 is xn's U whenever
// |U2| < 15, the only case in which its adjoint passes (at the clamp, xn holds
// +-15 and the adjoint is cut).
//
// Seven CTAs per SM (72 registers, some spilled to L1): the kernel waits on
// L2 gathers, and more resident warps hide them better than fewer spills do.
__global__ void __launch_bounds__(128, 7) adj_step_kernel(DevMesh<A> m, AdjMesh a, AdjStepBufs b,
                                                          const double *__restrict__ x, const double *__restrict__ xn,
                                                          const double *__restrict__ coef, StepParams p, int first,
                                                          int obs_row) {
    // launched with programmatic dependent launch: wait for the previous kernel's results
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = (gid >> 2) < m.C;
    const int c = valid ? gid >> 2 : m.C - 1, j = gid & 3;
    const int lane0 = (int)(threadIdx.x & 31) & ~3;
    double l[4], zg = 0.0;
    if (first) {
        for (int q = 0; q < 4; q++) l[q] = a.lam[4 * (size_t)c + q];
    } else {
        gather4(a, b.dir_in, b.so_in, b.sn_in, c, j, obs_row, l, zg);
    }
    const Vec4<double> xc = ldg4(x + 4 * (size_t)c);
    const double hv = xc.x, uv = xc.y, vv = xc.z;
    const double zbc = m.zbc[c];
    double whb = 0.0, wub = 0.0, wvb = 0.0;
    if (j == 0) {
        // ---- the update (UpdateCellKernel, functors.cu:717-784, variant H): forward values, then its reverse
        const double HM1 = p.hm1, HM2 = p.hm2;
        const double dta = m.dta[c];
        const Vec4<double> xn4 = ldg4(xn + 4 * (size_t)c);
        const double h2 = xn4.x, u2 = xn4.y, v2 = xn4.z;
        double h2b = l[0] + l[3];   // Z2 = H2 + ZBC
        double hb = 0.0, ub = 0.0, vb = 0.0, fncb = 0.0;
        if (h2 > HM2) {
            const UpdateCoef k = ld_coef(coef + UPDATE_COEF * (size_t)c);
            const double ue = fabs(u2) < 15.0 ? l[1] : 0.0;
            const double ve = fabs(v2) < 15.0 ? l[2] : 0.0;
            const double nub = ue * k.ih2, nvb = ve * k.ih2;
            h2b -= (ue * u2 + ve * v2) * k.ih2;
            hb += nub * uv + nvb * vv;
            ub += nub * (hv - k.dtw);
            vb += nvb * (hv - k.dtw);
            wub -= nub * dta;
            wvb -= nvb * dta;
            const double dtwb = -(nub * uv + nvb * vv);
            fncb += dtwb * k.d_fnc;
            hb += dtwb * k.d_h;
            ub += dtwb * k.d_s * uv;
            vb += dtwb * k.d_s * vv;
        } else if (h2 > HM1) {
            if (fabs(uv) < K::VMIN) ub += l[1];
            if (fabs(vv) < K::VMIN) vb += l[2];
        }
        if (h2 > HM1) { hb += h2b; whb -= h2b * dta; }
        if (valid) {
            stg4(b.dir_out + 4 * (size_t)c, hb, ub, vb, 0.0);
            a.fnc_g[c] += fncb;
            a.zbc_g[c] += l[3] + zg;
        }
    }
    whb = __shfl_sync(0xffffffffu, whb, lane0);
    wub = __shfl_sync(0xffffffffu, wub, lane0);
    wvb = __shfl_sync(0xffffffffu, wvb, lane0);
    if (!valid) return;
    // ---- lane j: slot 4c+j
    const size_t s = 4 * (size_t)c + j;
    double *so = b.so_out + ADJ_REC * s, *sno = b.sn_out + ADJ_REC * s;
    const uint8_t meta = a.meta4[s];
    if (meta == 0xFF) {
        st_rec(so, Adj5{0, 0, 0, 0, 0});
        st_rec(sno, Adj5{0, 0, 0, 0, 0});
        return;
    }
    const double cs = a.cs4[s], sn = a.sn4[s], side = a.side4[s];
    const double slcos = side * cs, slsin = side * sn;
    double fb[4];
    fb[0] = side * whb;
    fb[1] = slcos * wub + slsin * wvb;
    fb[2] = -slsin * wub + slcos * wvb;
    fb[3] = fb[1];
    SlotInA<A> in;
    in.own = CellStateA<A>{hv, uv, vv, xc.w, zbc};
    in.code = (int8_t)(meta & META_CODE);
    in.own_first = meta & META_OWN_FIRST;
    in.has_nb = meta & META_HAS_NB;
    const int nb = a.nbr4[s];
    if (in.has_nb) {
        const Vec4<double> xn4 = ldg4(x + 4 * (size_t)nb);
        in.nb = CellStateA<A>{xn4.x, xn4.y, xn4.z, xn4.w, m.zbc[nb]};
    }
    else
        in.nb = CellStateA<A>{0, 0, 0, 0, 0};
    in.cosj = cs; in.sinj = sn; in.side = side;
    auto fetch = [&]() {
        BoundaryInA<A> bi;
        const int row = m.bcell[c];
        if (row >= 0) {
            const size_t q = (size_t)p.jt * m.nb + row;
            bi.qt = m.bqt[q]; bi.dqt = m.bdqt[q]; bi.zt = m.bzt[q]; bi.dzt = m.bdzt[q];
            bi.top = m.btop[row]; bi.nhq1 = m.bnhq1[row];
            bi.zw = m.bzw + (size_t)row * m.nhq; bi.qw = m.bqw + (size_t)row * m.nhq;
        } else {
            bi.qt = bi.dqt = 0.0; bi.zt = bi.dzt = bi.top = 0.0; bi.nhq1 = 0;
            bi.zw = m.bzw + (size_t)m.nb * m.nhq; bi.qw = m.bqw + (size_t)m.nb * m.nhq;
        }
        bi.nhq = m.nhq;
        return bi;
    };
    Adj5 go{0, 0, 0, 0, 0}, gn{0, 0, 0, 0, 0};
    slot_rev(in, p, fetch, fb, go, gn, m.err);
    st_rec(so, go);
    st_rec(sno, gn);
}

// The adjoint of x_0 from step 0's contributions, into a.lam, with their bed terms.
__global__ void adj_gather_kernel(int C, AdjMesh a, const double *dir, const double *so, const double *sn) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = (gid >> 2) < C;
    const int c = valid ? gid >> 2 : C - 1, j = gid & 3;
    double l[4], zg;
    gather4(a, dir, so, sn, c, j, -1, l, zg);
    if (!valid || j != 0) return;
    for (int q = 0; q < 4; q++) a.lam[4 * (size_t)c + q] = l[q];
    a.zbc_g[c] += zg;
}

// lam = dL/dx_T (the last observation), zero elsewhere
__global__ void adj_seed_kernel(int C, AdjMesh a, int obs_row) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    double lh = 0.0;
    if (obs_row >= 0) {
        const int g = a.gauge_of[c];
        if (g >= 0) lh = 2.0 * a.res[(size_t)obs_row * a.ng + g];
    }
    a.lam[4 * (size_t)c] = lh;
    a.lam[4 * (size_t)c + 1] = 0.0;
    a.lam[4 * (size_t)c + 2] = 0.0;
    a.lam[4 * (size_t)c + 3] = 0.0;
}

// Initial state from the level (mesh.cpp:350-361) and its reverse.
__global__ void adj_init_state_kernel(int C, const double *__restrict__ z0, const double *__restrict__ u0,
                                      const double *__restrict__ v0, const double *__restrict__ zbc, double hm1,
                                      double *x) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    double h, z;
    if (z0[c] <= zbc[c]) { h = hm1; z = zbc[c] + hm1; }
    else { h = z0[c] - zbc[c]; z = z0[c]; }
    x[4 * (size_t)c] = h; x[4 * (size_t)c + 1] = u0[c]; x[4 * (size_t)c + 2] = v0[c]; x[4 * (size_t)c + 3] = z;
}
__global__ void adj_init_rev_kernel(int C, AdjMesh a, const double *__restrict__ z0, const double *__restrict__ zbc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    if (z0[c] <= zbc[c]) a.zbc_g[c] += a.lam[4 * (size_t)c + 3];   // Z0 = ZBC + HM1
    else a.zbc_g[c] -= a.lam[4 * (size_t)c];                        // H0 = Z0 - ZBC
}

__global__ void set_counter_kernel(long long *ctr, long long v) { *ctr = v; }

// The checkpoint and gauge kernels sit between step sequences of the forward
// and are chained to them by programmatic dependent launch: each waits for
// the previous kernel's results and lets the next one launch at once.

// the state before step t = *ctr into checkpoint t / k (when t is a multiple of k)
__global__ void ckpt_kernel(const double *S0, const double *S1, double *ckpt, const long long *ctr, int k,
                            size_t n) {
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
    const long long t = *ctr;
    if (t % k != 0) return;
    const double *src = (t & 1) ? S1 : S0;
    double *dst = ckpt + (size_t)(t / k) * n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// after t = *ctr steps, when t ends on an observation: the gauge depths into row t / obs_every - 1
__global__ void gauge_ctr_kernel(const double *S0, const double *S1, const int32_t *__restrict__ gcell, int ng,
                                 double *gd, const long long *ctr, int obs_every) {
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
    const long long t = *ctr;
    if (t == 0 || t % obs_every != 0) return;
    const double *S = (t & 1) ? S1 : S0;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < ng) gd[(size_t)(t / obs_every - 1) * ng + g] = S[4 * (size_t)gcell[g]];
}

// the gauge depths of state S (after a step that ends on an observation) into row `row`
__global__ void gauge_state_kernel(const double *S, const int32_t *__restrict__ gcell, int ng, double *gd, int row) {
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < ng) gd[(size_t)row * ng + g] = S[4 * (size_t)gcell[g]];
}

}  // namespace adj
}  // namespace hb

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct hb_adjoint {
    hb_handle *h = nullptr;
    int C = 0, T = 0, k = 0, obs_every = 0, ng = 0, nobs = 0;
    std::vector<void *> allocs;
    std::vector<int32_t> gauges_dev;        // gauge cells, device order
    int32_t *d_gcell = nullptr;
    double *d_ckpt = nullptr;               // [T/k + 1][C][4]
    double *d_seg[2] = {nullptr, nullptr};   // [k + 1][C][4] states of a segment (two segments in flight)
    double *d_terms = nullptr;              // [4C][4] slot terms of the step being recomputed
    double *d_coef[2] = {nullptr, nullptr}; // [k][C][UPDATE_COEF] update coefficients of a segment
    int recorded_seg = -1;                  // segment whose states the forward left in d_seg (-1: none)
    cudaStream_t recompute = nullptr;        // the recomputation, ahead of the reverse steps (highest priority)
    cudaStream_t reverse = nullptr;          // the reverse steps (lowest priority)
    cudaEvent_t ev_recomputed[2] = {nullptr, nullptr}, ev_reversed[2] = {nullptr, nullptr};
    double *d_gd = nullptr;                 // [nobs][ng] gauge depths of the forward
    double *d_obs = nullptr;                // [nobs][ng]
    double *d_res = nullptr;                // [nobs][ng]
    double *d_z0 = nullptr, *d_u0 = nullptr, *d_v0 = nullptr;   // initial level and velocities (device order)
    double *d_dir[2] = {nullptr, nullptr};  // [C][4] the update's direct terms, by step parity
    double *d_so[2] = {nullptr, nullptr};   // [4C][ADJ_REC] slots' contributions to their own cells
    double *d_sn[2] = {nullptr, nullptr};   // [4C][ADJ_REC] slots' contributions to their neighbours
    hb::adj::AdjMesh am{};
    cudaGraphExec_t fwd_graph = nullptr;    // k forward steps with checkpoint and gauge kernels
    cudaGraphExec_t fwd_graph_multi = nullptr;   // 100 / k such segments
    // the whole backward pass (recomputation and reverse steps on their two
    // streams), one graph for a backward that follows its forward (whose last
    // segment is in place) and one for a repeated backward
    cudaGraphExec_t bwd_graph[2] = {nullptr, nullptr};
    bool forward_done = false;
    ~hb_adjoint() {
        if (fwd_graph) cudaGraphExecDestroy(fwd_graph);
        if (fwd_graph_multi) cudaGraphExecDestroy(fwd_graph_multi);
        for (auto &g : bwd_graph)
            if (g) cudaGraphExecDestroy(g);
        for (int q = 0; q < 2; q++) {
            if (ev_recomputed[q]) cudaEventDestroy(ev_recomputed[q]);
            if (ev_reversed[q]) cudaEventDestroy(ev_reversed[q]);
        }
        if (recompute) cudaStreamDestroy(recompute);
        if (reverse) cudaStreamDestroy(reverse);
        for (void *p : allocs) cudaFree(p);
    }
};

namespace {

template <class T>
int adj_alloc(hb_adjoint *a, T **dst, size_t count) {
    void *p = nullptr;
    const size_t n = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) return hb::set_error(HB_E_NOMEM, "adjoint: cudaMalloc(%zu): %s", n, cudaGetErrorString(e));
    a->allocs.push_back(p);
    HB_CUDA_RET(cudaMemset(p, 0, n));
    *dst = (T *)p;
    return HB_OK;
}
template <class T>
int adj_upload(hb_adjoint *a, T **dst, const std::vector<T> &v) {
    TRY(adj_alloc(a, dst, v.size()));
    if (!v.empty()) HB_CUDA_RET(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return HB_OK;
}

hb::StepParams step_params(const hb_handle *h, long long step) {
    const hb::Scenario &sc = h->scn[0];
    hb::StepParams p;
    p.hm1 = sc.hm1; p.hm2 = sc.hm2; p.jl = sc.jl; p.dt = sc.dt;
    p.jt = (int)(step / sc.per_day);
    p.kt = 1 + (int)(step % sc.per_day);
    return p;
}

}  // namespace

extern "C" int hb_adjoint_create(hb_handle *h, const int32_t *gauges, int32_t ngauges, int32_t obs_every,
                                 int32_t nsteps, int32_t checkpoint_every, hb_adjoint **out) {
    if (!h || !out || !gauges || ngauges <= 0 || obs_every <= 0 || nsteps <= 0 || checkpoint_every <= 0)
        return hb::set_error(HB_E_INVALID, "hb_adjoint_create: bad argument");
    *out = nullptr;
    if (h->opt.precision != HB_FP64 || h->opt.variant != HB_VARIANT_H || h->opt.layout != HB_LAYOUT_EDGE ||
        h->opt.persistent || h->scn.size() != 1)
        return hb::set_error(HB_E_INVALID,
                             "hb_adjoint_create: needs a single-mesh fp64 variant-H edge-layout handle (not persistent)");
    if (nsteps > h->step_limit()) return hb::set_error(HB_E_INVALID, "hb_adjoint_create: %d steps beyond the boundary tables", nsteps);
    const hb::Scenario &sc = h->scn[0];
    const int C = sc.cells;
    for (int i = 0; i < ngauges; i++)
        if (gauges[i] < 0 || gauges[i] >= C) return hb::set_error(HB_E_INVALID, "hb_adjoint_create: gauge %d out of range", gauges[i]);
    {   // one gauge per cell: the reverse sweep and the fused forward map each cell to one gauge
        std::vector<char> seen(C, 0);
        for (int i = 0; i < ngauges; i++) {
            if (seen[gauges[i]]) return hb::set_error(HB_E_INVALID, "hb_adjoint_create: cell %d is a gauge twice", gauges[i]);
            seen[gauges[i]] = 1;
        }
    }
    // per-slot geometry, codes and facing slots (device order); codes without a reverse are rejected
    std::vector<double> cs4(4 * (size_t)C, 0.0), sn4(4 * (size_t)C, 0.0), side4(4 * (size_t)C, 0.0);
    std::vector<int32_t> nbr4(4 * (size_t)C, -1), mirror4(4 * (size_t)C, -1);
    std::vector<uint8_t> meta4(4 * (size_t)C, 0xFF);
    auto a = new hb_adjoint();
    a->h = h; a->C = C; a->T = nsteps; a->k = checkpoint_every; a->obs_every = obs_every; a->ng = ngauges;
    a->nobs = nsteps / obs_every;
    const int nrec = h->m64.nrecords;
    std::vector<int4> rix(nrec);
    std::vector<uint8_t> rmeta(nrec);
    std::vector<double> rgeo(4 * (size_t)nrec);
    int st = HB_OK;
    auto fail = [&](int s) { delete a; return s; };
    if (cudaMemcpy(rix.data(), h->m64.rix, nrec * sizeof(int4), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(rmeta.data(), h->m64.rmeta, nrec, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(rgeo.data(), h->m64.rgeo, 4 * (size_t)nrec * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(hb::set_error(HB_E_CUDA, "hb_adjoint_create: reading the device mesh"));
    for (int r = 0; r < nrec; r++) {
        const int4 ix = rix[r];
        const int code = rmeta[r] & hb::META_CODE;
        if (code != hb::CODE_ZERO && code != hb::CODE_K4 && code != hb::CODE_K10 && code != hb::CODE_K1)
            return fail(hb::set_error(HB_E_INVALID, "hb_adjoint_create: boundary code %d has no reverse here (KLAS 0, 1, 4, 10 only)", code));
        const double *g = &rgeo[4 * (size_t)r];
        cs4[ix.z] = g[0]; sn4[ix.z] = g[1]; side4[ix.z] = g[2]; nbr4[ix.z] = ix.y; meta4[ix.z] = rmeta[r];
        if (ix.w >= 0) {
            // the other slot of a mirror pair: reversed normal, neighbour a, not the lower-numbered side
            cs4[ix.w] = -g[0]; sn4[ix.w] = -g[1]; side4[ix.w] = g[2]; nbr4[ix.w] = ix.x;
            meta4[ix.w] = (uint8_t)(hb::CODE_ZERO | hb::META_HAS_NB);
        }
    }
    // The gather of cell c reads the neighbours' slots that face c through
    // mirror4 of c's own slots: a one-to-one pairing of the slots of c that
    // face a neighbour with the neighbour's slots that face c.
    std::vector<char> claimed(4 * (size_t)C, 0);
    for (int c = 0; c < C; c++)
        for (int j = 0; j < 4; j++) {
            const size_t s = 4 * (size_t)c + j;
            const int nb = nbr4[s];
            if (meta4[s] == 0xFF || nb < 0) continue;
            for (int q = 0; q < 4; q++) {
                const size_t t = 4 * (size_t)nb + q;
                if (nbr4[t] == c && meta4[t] != 0xFF && !claimed[t]) { mirror4[s] = (int32_t)t; claimed[t] = 1; break; }
            }
            if (mirror4[s] < 0) return fail(hb::set_error(HB_E_BADMESH, "hb_adjoint_create: cell %d slot %d has no facing slot", c, j));
        }
    std::vector<int32_t> gauge_of(C, -1);
    a->gauges_dev.resize(ngauges);
    for (int g = 0; g < ngauges; g++) {
        const int d = sc.inv[gauges[g]];
        a->gauges_dev[g] = d;
        gauge_of[d] = g;
    }
    hb::adj::AdjMesh &am = a->am;
    double *dp;
    int32_t *ip;
    uint8_t *up;
    if ((st = adj_upload(a, &dp, cs4)) != HB_OK) return fail(st);
    am.cs4 = dp;
    if ((st = adj_upload(a, &dp, sn4)) != HB_OK) return fail(st);
    am.sn4 = dp;
    if ((st = adj_upload(a, &dp, side4)) != HB_OK) return fail(st);
    am.side4 = dp;
    if ((st = adj_upload(a, &ip, nbr4)) != HB_OK) return fail(st);
    am.nbr4 = ip;
    if ((st = adj_upload(a, &ip, mirror4)) != HB_OK) return fail(st);
    am.mirror4 = ip;
    if ((st = adj_upload(a, &up, meta4)) != HB_OK) return fail(st);
    am.meta4 = up;
    if ((st = adj_upload(a, &ip, gauge_of)) != HB_OK) return fail(st);
    am.gauge_of = ip;
    if ((st = adj_upload(a, &a->d_gcell, a->gauges_dev)) != HB_OK) return fail(st);
    for (int q = 0; q < 2; q++) {
        if ((st = adj_alloc(a, &a->d_dir[q], 4 * (size_t)C)) != HB_OK) return fail(st);
        if ((st = adj_alloc(a, &a->d_so[q], 4 * hb::adj::ADJ_REC * (size_t)C)) != HB_OK) return fail(st);
        if ((st = adj_alloc(a, &a->d_sn[q], 4 * hb::adj::ADJ_REC * (size_t)C)) != HB_OK) return fail(st);
    }
    if ((st = adj_alloc(a, &am.fnc_g, C)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &am.zbc_g, C)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &am.lam, 4 * (size_t)C)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &a->d_res, (size_t)std::max(a->nobs, 1) * ngauges)) != HB_OK) return fail(st);
    am.res = a->d_res;
    am.ng = ngauges;
    am.obs_every = obs_every;
    const int nck = nsteps / checkpoint_every + 1;
    if ((st = adj_alloc(a, &a->d_ckpt, (size_t)nck * 4 * C)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &a->d_terms, 16 * (size_t)C)) != HB_OK) return fail(st);
    for (int q = 0; q < 2; q++) {
        if ((st = adj_alloc(a, &a->d_seg[q], (size_t)(checkpoint_every + 1) * 4 * C)) != HB_OK) return fail(st);
        if ((st = adj_alloc(a, &a->d_coef[q], (size_t)checkpoint_every * hb::UPDATE_COEF * C)) != HB_OK)
            return fail(st);
        if (cudaEventCreateWithFlags(&a->ev_recomputed[q], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&a->ev_reversed[q], cudaEventDisableTiming) != cudaSuccess)
            return fail(hb::set_error(HB_E_CUDA, "hb_adjoint_create: cudaEventCreate failed"));
    }
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&a->recompute, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&a->reverse, cudaStreamNonBlocking, least) != cudaSuccess)
        return fail(hb::set_error(HB_E_CUDA, "hb_adjoint_create: cudaStreamCreate failed"));
    if ((st = adj_alloc(a, &a->d_gd, (size_t)std::max(a->nobs, 1) * ngauges)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &a->d_obs, (size_t)std::max(a->nobs, 1) * ngauges)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &a->d_z0, C)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &a->d_u0, C)) != HB_OK) return fail(st);
    if ((st = adj_alloc(a, &a->d_v0, C)) != HB_OK) return fail(st);
    *out = a;
    return HB_OK;
}

extern "C" int hb_adjoint_destroy(hb_adjoint *a) {
    delete a;
    return HB_OK;
}

extern "C" int hb_adjoint_set_parameters(hb_adjoint *a, const double *manning_n, const double *zbc) {
    if (!a) return hb::set_error(HB_E_INVALID, "null adjoint");
    const hb::Scenario &sc = a->h->scn[0];
    const int C = a->C;
    std::vector<double> v(C);
    if (manning_n) {
        for (int i = 0; i < C; i++) { const double n = manning_n[sc.perm[i]]; v[i] = 9.81 * n * n; }
        HB_CUDA_RET(cudaMemcpy(const_cast<double *>(a->h->m64.fnc), v.data(), C * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (zbc) {
        for (int i = 0; i < C; i++) v[i] = zbc[sc.perm[i]];
        HB_CUDA_RET(cudaMemcpy(const_cast<double *>(a->h->m64.zbc), v.data(), C * sizeof(double), cudaMemcpyHostToDevice));
    }
    a->forward_done = false;
    return HB_OK;
}

extern "C" int hb_adjoint_set_initial(hb_adjoint *a, const double *Z0, const double *U0, const double *V0) {
    if (!a || !Z0 || !U0 || !V0) return hb::set_error(HB_E_INVALID, "hb_adjoint_set_initial: bad argument");
    const hb::Scenario &sc = a->h->scn[0];
    const int C = a->C;
    std::vector<double> v(C);
    const double *src[3] = {Z0, U0, V0};
    double *dst[3] = {a->d_z0, a->d_u0, a->d_v0};
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < C; i++) v[i] = src[k][sc.perm[i]];
        HB_CUDA_RET(cudaMemcpy(dst[k], v.data(), C * sizeof(double), cudaMemcpyHostToDevice));
    }
    a->forward_done = false;
    return HB_OK;
}

extern "C" int hb_adjoint_set_observations(hb_adjoint *a, const double *obs) {
    if (!a || !obs) return hb::set_error(HB_E_INVALID, "hb_adjoint_set_observations: bad argument");
    HB_CUDA_RET(cudaMemcpy(a->d_obs, obs, (size_t)a->nobs * a->ng * sizeof(double), cudaMemcpyHostToDevice));
    return HB_OK;
}

extern "C" int hb_adjoint_forward(hb_adjoint *a, double *loss, double *gauge_depths, void *stream) {
    NvtxRange nvtx_("hb_adjoint_forward");
    if (!a) return hb::set_error(HB_E_INVALID, "null adjoint");
    hb_handle *h = a->h;
    cudaStream_t st = (cudaStream_t)stream;
    const int C = a->C;
    const size_t S4 = 4 * (size_t)C;
    hb::adj::adj_init_state_kernel<<<(C + 255) / 256, 256, 0, st>>>(C, a->d_z0, a->d_u0, a->d_v0, h->m64.zbc,
                                                                     h->scn[0].hm1, h->m64.S[0]);
    HB_CUDA_RET(cudaGetLastError());
    hb::adj::set_counter_kernel<<<1, 1, 0, st>>>(h->d_ctr, 0);
    HB_CUDA_RET(cudaMemsetAsync(h->d_err, 0, sizeof(uint32_t), st));
    h->steps_done = 0;
    a->recorded_seg = -1;
    // forward segments: checkpoint at each segment's start, gauge depths
    // after every step that ends on an observation (positions fixed when k is
    // a multiple of obs_every, otherwise after every step)
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    // Fused form (plain fp64 edge-layout handles): the cell kernel of each
    // step writes the checkpoints and gauge depths itself (hb::DevMesh's
    // adjoint outputs), so a run of segments is one step sequence with no
    // kernels between the steps; checkpoint 0 is copied once up front.
    const bool fused = hb_steps_take_mesh(h);
    hb::DevMesh<hb::F64Exact> mk = h->m64;
    mk.ckpt = a->d_ckpt;
    mk.ckpt_every = a->k;
    mk.gauge_of = a->am.gauge_of;
    mk.gauge_out = a->d_gd;
    mk.obs_every = a->obs_every;
    mk.ngauge = a->ng;
    if (fused) {
        cudaLaunchConfig_t c0{};
        c0.gridDim = dim3(64);
        c0.blockDim = dim3(256);
        c0.stream = st;
        c0.attrs = attr;
        c0.numAttrs = 1;
        HB_CUDA_RET(cudaLaunchKernelEx(&c0, hb::adj::ckpt_kernel, (const double *)h->m64.S[0],
                                       (const double *)h->m64.S[1], a->d_ckpt, (const long long *)h->d_ctr, a->k, S4));
    }
    // nsegs k-step segments from a step that is a multiple of k
    auto enqueue = [&](int nsegs, cudaStream_t s) -> int {
        if (fused) return hb_enqueue_steps_mesh(h, mk, nsegs * a->k, s);
        const double *S0 = h->m64.S[0], *S1 = h->m64.S[1];
        cudaLaunchConfig_t ck{};
        ck.gridDim = dim3(64);
        ck.blockDim = dim3(256);
        ck.stream = s;
        ck.attrs = attr;
        ck.numAttrs = 1;
        cudaLaunchConfig_t gk = ck;
        gk.gridDim = dim3((unsigned)((a->ng + 127) / 128));
        gk.blockDim = dim3(128);
        for (int q = 0; q < nsegs; q++) {
            HB_CUDA_RET(cudaLaunchKernelEx(&ck, hb::adj::ckpt_kernel, S0, S1, a->d_ckpt, (const long long *)h->d_ctr,
                                           a->k, S4));
            // runs of steps up to each observation: one multi-step launch sequence each
            for (int i = 0; i < a->k;) {
                int m = a->k - i;
                if (a->k % a->obs_every == 0) m = std::min(m, a->obs_every - i % a->obs_every);
                else m = 1;
                TRY(hb_enqueue_steps(h, m, s));
                i += m;
                HB_CUDA_RET(cudaLaunchKernelEx(&gk, hb::adj::gauge_ctr_kernel, S0, S1, (const int32_t *)a->d_gcell,
                                               a->ng, a->d_gd, (const long long *)h->d_ctr, a->obs_every));
            }
        }
        return HB_OK;
    };
    auto capture = [&](int nsegs, cudaGraphExec_t *exec) -> int {
        cudaStream_t cap;
        HB_CUDA_RET(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        HB_CUDA_RET(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue(nsegs, cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc != HB_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return hb::set_error(HB_E_CUDA, "adjoint forward capture: %s", cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            *exec = nullptr;
            return hb::set_error(HB_E_CUDA, "adjoint forward graph: %s", cudaGetErrorString(ei));
        }
        return HB_OK;
    };
    // Segments 0 .. nseg-2 replay captured graphs: one of G = 100 / k
    // segments (about 100 steps) where it fits, one segment otherwise.  The
    // last segment (k steps or the remainder) is stepped into the segment
    // buffer with its update coefficients, as the backward pass would
    // recompute it, so the backward starts reversing at once.
    const int nseg = (a->T + a->k - 1) / a->k;
    const int ngraph = nseg - 1;
    const int G = std::max(1, 100 / a->k);
    int done = 0;
    if (G > 1 && ngraph >= G) {
        if (!a->fwd_graph_multi) TRY(capture(G, &a->fwd_graph_multi));
        for (; done + G <= ngraph; done += G) HB_CUDA_RET(cudaGraphLaunch(a->fwd_graph_multi, st));
    }
    if (done < ngraph) {
        if (!a->fwd_graph) TRY(capture(1, &a->fwd_graph));
        for (; done < ngraph; done++) HB_CUDA_RET(cudaGraphLaunch(a->fwd_graph, st));
    }
    {
        const int sgi = nseg - 1, t0 = sgi * a->k, len = a->T - t0, b = sgi & 1;
        cudaLaunchConfig_t ck{};
        ck.gridDim = dim3(64);
        ck.blockDim = dim3(256);
        ck.stream = st;
        ck.attrs = attr;
        ck.numAttrs = 1;
        cudaLaunchConfig_t gk = ck;
        gk.gridDim = dim3((unsigned)((a->ng + 127) / 128));
        gk.blockDim = dim3(128);
        // (fused: the segment's checkpoint was written by the step before it, or up front)
        if (!fused)
            HB_CUDA_RET(cudaLaunchKernelEx(&ck, hb::adj::ckpt_kernel, (const double *)h->m64.S[0],
                                           (const double *)h->m64.S[1], a->d_ckpt, (const long long *)h->d_ctr, a->k,
                                           S4));
        for (int i = 0; i < len; i++) {
            const double *in = i == 0 ? h->m64.S[t0 & 1] : a->d_seg[b] + (size_t)i * S4;
            double *out = a->d_seg[b] + (size_t)(i + 1) * S4;
            TRY(hb_forward_step_into(h, t0, i, in, out, a->d_terms, a->d_coef[b] + (size_t)i * hb::UPDATE_COEF * C,
                                     (int)(i == len - 1), st));
            const int t = t0 + i + 1;
            if (t % a->obs_every == 0)
                HB_CUDA_RET(cudaLaunchKernelEx(&gk, hb::adj::gauge_state_kernel, (const double *)out,
                                               (const int32_t *)a->d_gcell, a->ng, a->d_gd, t / a->obs_every - 1));
        }
        // the handle's state and counter after the rollout
        HB_CUDA_RET(cudaMemcpyAsync(h->m64.S[a->T & 1], a->d_seg[b] + (size_t)len * S4, S4 * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st));
        hb::adj::set_counter_kernel<<<1, 1, 0, st>>>(h->d_ctr, a->T);
        HB_CUDA_RET(cudaGetLastError());
        a->recorded_seg = sgi;
    }
    h->steps_done = a->T;
    HB_CUDA_RET(cudaStreamSynchronize(st));
    uint32_t bits = 0;
    HB_CUDA_RET(cudaMemcpy(&bits, h->d_err, sizeof bits, cudaMemcpyDeviceToHost));
    if (bits) return hb::set_error(HB_E_NONFINITE, "hb_adjoint_forward: device error bits 0x%x", bits);
    const size_t no = (size_t)a->nobs * a->ng;
    std::vector<double> gd(no), ob(no), res(no);
    HB_CUDA_RET(cudaMemcpy(gd.data(), a->d_gd, no * sizeof(double), cudaMemcpyDeviceToHost));
    HB_CUDA_RET(cudaMemcpy(ob.data(), a->d_obs, no * sizeof(double), cudaMemcpyDeviceToHost));
    double L = 0.0;
    for (size_t i = 0; i < no; i++) { res[i] = gd[i] - ob[i]; L += res[i] * res[i]; }
    HB_CUDA_RET(cudaMemcpy(a->d_res, res.data(), no * sizeof(double), cudaMemcpyHostToDevice));
    if (loss) *loss = L;
    if (gauge_depths) memcpy(gauge_depths, gd.data(), no * sizeof(double));
    a->forward_done = true;
    return HB_OK;
}

namespace {

// The backward pass's device work, on the reverse stream `st` and the
// recompute stream (forked from and joined back to `st`).  have_last: the
// forward left the last segment's states and coefficients in place.
int enqueue_backward(hb_adjoint *a, bool have_last, cudaStream_t st, std::vector<cudaEvent_t> &temp_events) {
    hb_handle *h = a->h;
    const int C = a->C;
    const size_t S4 = 4 * (size_t)C;
    hb::adj::AdjMesh am = a->am;
    HB_CUDA_RET(cudaMemsetAsync(am.fnc_g, 0, C * sizeof(double), st));
    HB_CUDA_RET(cudaMemsetAsync(am.zbc_g, 0, C * sizeof(double), st));
    const int cb = (C + 255) / 256;
    hb::adj::adj_seed_kernel<<<cb, 256, 0, st>>>(C, am, a->T % a->obs_every == 0 ? a->T / a->obs_every - 1 : -1);
    HB_CUDA_RET(cudaGetLastError());
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)((4 * C + 127) / 128));
    cfg.blockDim = dim3(128);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int nseg = (a->T + a->k - 1) / a->k;
    // Segment sgi's states and update coefficients are recomputed on the
    // recompute stream into buffer sgi & 1, one segment ahead of the reverse
    // steps on `st`: recompute(sgi - 1) overlaps reverse(sgi).  Each step's
    // slot terms only pass through d_terms on the recompute stream.  Events
    // order each buffer's reuse.  The reverse kernels do not read the step
    // counter or any other array the forward kernels write besides the
    // segment buffers.
    cudaStream_t rs = a->recompute;
    cudaEvent_t fork = nullptr, join = nullptr;
    HB_CUDA_RET(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    temp_events.push_back(fork);
    HB_CUDA_RET(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    temp_events.push_back(join);
    HB_CUDA_RET(cudaEventRecord(fork, st));
    HB_CUDA_RET(cudaStreamWaitEvent(rs, fork, 0));   // after this pass's earlier work on st
    bool reversed_once[2] = {false, false};
    // state i of segment sgi: its checkpoint, then the segment buffer
    auto seg_state = [&](int sgi, int i) -> const double * {
        return i == 0 ? a->d_ckpt + (size_t)sgi * S4 : a->d_seg[sgi & 1] + (size_t)i * S4;
    };
    auto issue_recompute = [&](int sgi) -> int {
        const int b = sgi & 1;
        const int t0 = sgi * a->k, len = std::min(t0 + a->k, a->T) - t0;
        if (reversed_once[b]) HB_CUDA_RET(cudaStreamWaitEvent(rs, a->ev_reversed[b], 0));
        hb::adj::set_counter_kernel<<<1, 1, 0, rs>>>(h->d_ctr, t0);
        for (int i = 0; i < len; i++)
            TRY(hb_forward_step_into(h, t0, i, seg_state(sgi, i), a->d_seg[b] + (size_t)(i + 1) * S4, a->d_terms,
                                     a->d_coef[b] + (size_t)i * hb::UPDATE_COEF * C, 0, rs));
        HB_CUDA_RET(cudaEventRecord(a->ev_recomputed[b], rs));
        return HB_OK;
    };
    if (!have_last) TRY(issue_recompute(nseg - 1));
    for (int sgi = nseg - 1; sgi >= 0; sgi--) {
        const int b = sgi & 1;
        const int t0 = sgi * a->k, len = std::min(t0 + a->k, a->T) - t0;
        if (sgi > 0) TRY(issue_recompute(sgi - 1));
        if (sgi != nseg - 1 || !have_last) HB_CUDA_RET(cudaStreamWaitEvent(st, a->ev_recomputed[b], 0));
        for (int i = len - 1; i >= 0; i--) {
            const int t = t0 + i;
            const hb::StepParams p = step_params(h, t);
            const int w = t & 1;
            const hb::adj::AdjStepBufs bufs{a->d_dir[w ^ 1], a->d_so[w ^ 1], a->d_sn[w ^ 1],
                                            a->d_dir[w], a->d_so[w], a->d_sn[w]};
            const int row = (t + 1 < a->T && (t + 1) % a->obs_every == 0) ? (t + 1) / a->obs_every - 1 : -1;
            const double *xs = seg_state(sgi, i), *xn = a->d_seg[b] + (size_t)(i + 1) * S4;
            const double *cf = a->d_coef[b] + (size_t)i * hb::UPDATE_COEF * C;
            HB_CUDA_RET(cudaLaunchKernelEx(&cfg, hb::adj::adj_step_kernel, h->m64, am, bufs, xs, xn, cf, p,
                                           (int)(t == a->T - 1), row));
        }
        HB_CUDA_RET(cudaEventRecord(a->ev_reversed[b], st));
        reversed_once[b] = true;
    }
    // the recompute stream's work is all joined by now; join it explicitly too
    HB_CUDA_RET(cudaEventRecord(join, rs));
    HB_CUDA_RET(cudaStreamWaitEvent(st, join, 0));
    // the adjoint of x_0 (step 0 wrote copy 0)
    hb::adj::adj_gather_kernel<<<(4 * C + 127) / 128, 128, 0, st>>>(C, am, a->d_dir[0], a->d_so[0], a->d_sn[0]);
    HB_CUDA_RET(cudaGetLastError());
    hb::adj::adj_init_rev_kernel<<<cb, 256, 0, st>>>(C, am, a->d_z0, h->m64.zbc);
    HB_CUDA_RET(cudaGetLastError());
    // leave the handle's counter where the forward left it
    hb::adj::set_counter_kernel<<<1, 1, 0, st>>>(h->d_ctr, a->T);
    return HB_OK;
}

// Captures enqueue_backward on the reverse stream into an executable graph
// that keeps the recompute stream's higher priority per node.
int capture_backward(hb_adjoint *a, bool have_last, cudaGraphExec_t *exec) {
    cudaStream_t st = a->reverse;
    std::vector<cudaEvent_t> temp;
    HB_CUDA_RET(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_backward(a, have_last, st, temp);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    for (cudaEvent_t ev : temp) cudaEventDestroy(ev);
    if (rc != HB_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return hb::set_error(HB_E_CUDA, "adjoint backward capture: %s", cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiateWithFlags(exec, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        *exec = nullptr;
        return hb::set_error(HB_E_CUDA, "adjoint backward graph: %s", cudaGetErrorString(ei));
    }
    return HB_OK;
}

}  // namespace

extern "C" int hb_adjoint_backward(hb_adjoint *a, double *grad_n, double *grad_zbc, void *stream) {
    NvtxRange nvtx_("hb_adjoint_backward");
    if (!a) return hb::set_error(HB_E_INVALID, "null adjoint");
    if (!a->forward_done) return hb::set_error(HB_E_INVALID, "hb_adjoint_backward: run hb_adjoint_forward first");
    hb_handle *h = a->h;
    // The reverse steps run on the adjoint's own lowest-priority stream and
    // the recomputation of the next segment on its highest-priority one, both
    // joined to the caller's stream.  The recomputation is a chain of small
    // kernels; given priority, its blocks start as soon as they are ready
    // instead of queueing behind the reverse grids, which fill the rest of
    // the GPU (measured: backward 19.4 -> 17.1 ms on the 24K-cell, 1000-step
    // case; the other way round, 21.1 ms).  The pass is one graph, captured
    // on first use (per kind of pass) and replayed after: its thousands of
    // launches then cost no host time each.
    cudaStream_t user = (cudaStream_t)stream;
    cudaStream_t st = a->reverse;
    {
        cudaEvent_t join = nullptr;
        HB_CUDA_RET(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
        HB_CUDA_RET(cudaEventRecord(join, user));
        HB_CUDA_RET(cudaStreamWaitEvent(st, join, 0));
        cudaEventDestroy(join);
    }
    const int C = a->C;
    const hb::adj::AdjMesh am = a->am;
    const int nseg = (a->T + a->k - 1) / a->k;
    // the forward left the last segment's states and coefficients in place
    const bool have_last = a->recorded_seg == nseg - 1;
    cudaGraphExec_t &ge = a->bwd_graph[have_last ? 1 : 0];
    if (!ge) TRY(capture_backward(a, have_last, &ge));
    HB_CUDA_RET(cudaGraphLaunch(ge, st));
    a->recorded_seg = -1;   // the segment buffers were reused
    {
        cudaEvent_t done = nullptr;
        HB_CUDA_RET(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        HB_CUDA_RET(cudaEventRecord(done, st));
        HB_CUDA_RET(cudaStreamWaitEvent(user, done, 0));
        cudaEventDestroy(done);
    }
    HB_CUDA_RET(cudaStreamSynchronize(st));
    uint32_t bits = 0;
    HB_CUDA_RET(cudaMemcpy(&bits, h->d_err, sizeof bits, cudaMemcpyDeviceToHost));
    if (bits) return hb::set_error(HB_E_UNDEFINED_REF, "hb_adjoint_backward: device error bits 0x%x", bits);
    const hb::Scenario &sc = h->scn[0];
    std::vector<double> g(C), fnc(C);
    if (grad_n) {
        HB_CUDA_RET(cudaMemcpy(g.data(), am.fnc_g, C * sizeof(double), cudaMemcpyDeviceToHost));
        HB_CUDA_RET(cudaMemcpy(fnc.data(), h->m64.fnc, C * sizeof(double), cudaMemcpyDeviceToHost));
        // FNC = 9.81 n^2: dL/dn = dL/dFNC * 2 * 9.81 * n, n = sqrt(FNC / 9.81)
        for (int i = 0; i < C; i++) grad_n[sc.perm[i]] = g[i] * 2.0 * 9.81 * std::sqrt(fnc[i] / 9.81);
    }
    if (grad_zbc) {
        HB_CUDA_RET(cudaMemcpy(g.data(), am.zbc_g, C * sizeof(double), cudaMemcpyDeviceToHost));
        for (int i = 0; i < C; i++) grad_zbc[sc.perm[i]] = g[i];
    }
    return HB_OK;
}
