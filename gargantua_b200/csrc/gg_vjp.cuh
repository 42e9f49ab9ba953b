// gg_vjp.cuh -- vector-Jacobian products of one Kerr right-hand side
// a^mu(r, theta, w; spin) = kerr_contract(kerr_geometry(M, a, r, sin, cos), w)
// (the geodesic equation of kerr.rs:154-204, grouped as the trace kernels do): given
// a cotangent kb of a, the products kb . da/dr, kb . da/dtheta, kb . da/dw^m
// and kb . da/da.  Two forms of the same derivatives: dual numbers (forward
// mode, straight from the templated physics) and a hand-written reverse pass
// through the geometry and the contraction.  The adjoint's backward uses one
// of them (GG_ADJ_HAND_VJP); gg_check_kerr_vjp runs both on the same points.
#pragma once

#include "gg_device.cuh"
#include "gg_dual.cuh"

namespace gg {

// Vector-Jacobian product of one Kerr right-hand side a^mu(r, theta, w; spin)
// with the cotangent kb: Xr, Xth, W[4] and (accumulated) *ga are kb . da/dr,
// da/dtheta, da/dw^m and da/dspin.  The geometry depends on (r, theta, spin)
// only and the contraction is quadratic in w, so the r, theta and spin columns
// come from a 3-direction dual evaluation with w held constant, and the w
// columns from a 4-direction dual of the contraction alone with the
// geometry's values held constant.  Each direction's arithmetic is the one
// a single 7-direction evaluation would do (the terms dropped are exact
// zeros), at about half its cost.
GG_DEV void kerr_rhs_vjp_dual(double M, double spin, double r, double th, const double w[4],
                              const double kb[4], double* Xr, double* Xth, double W[4], double* ga) {
  Dual<3> s, c;
  sincos(Dual<3>::var(th, 1), &s, &c);
  const KerrGeo<Dual<3>> G =
      kerr_geometry<Dual<3>>(Dual<3>(M), Dual<3>::var(spin, 2), Dual<3>::var(r, 0), s, c);
  Dual<3> w3[4], acc3[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) w3[i] = Dual<3>(w[i]);
  kerr_contract<Dual<3>>(G, w3, acc3);
  KerrGeo<Dual<4>> Gv;  // the geometry's values, constant in w
  Gv.dtt_r = G.dtt_r.v;
  Gv.dtt_th = G.dtt_th.v;
  Gv.drr_r = G.drr_r.v;
  Gv.drr_th = G.drr_th.v;
  Gv.dthth_r = G.dthth_r.v;
  Gv.dthth_th = G.dthth_th.v;
  Gv.dphph_r = G.dphph_r.v;
  Gv.dphph_th = G.dphph_th.v;
  Gv.dtph_r = G.dtph_r.v;
  Gv.dtph_th = G.dtph_th.v;
  Gv.gtt = G.gtt.v;
  Gv.gtph = G.gtph.v;
  Gv.gphph = G.gphph.v;
  Gv.hrr = G.hrr.v;
  Gv.hthth = G.hthth.v;
  Dual<4> w4[4], acc4[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) w4[i] = Dual<4>::var(w[i], i);
  kerr_contract<Dual<4>>(Gv, w4, acc4);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    *Xr += acc3[i].d[0] * kb[i];
    *Xth += acc3[i].d[1] * kb[i];
#pragma unroll
    for (int m = 0; m < 4; ++m) W[m] += acc4[i].d[m] * kb[i];
    *ga += acc3[i].d[2] * kb[i];
  }
}

// The same products by reverse accumulation: the geometry's base quantities
// and the contraction's intermediates forward, then their cotangents in
// reverse order.  Term by term against kerr_geometry / kerr_contract: 1/Sigma,
// 1/Delta and 1/sin^2 come from the one reciprocal the geometry takes, and
// their cotangents go back through d(1/x) = -(1/x)^2 dx.  One sweep back
// through the scalar terms, where the dual form carries three and four
// derivative directions through every product.
GG_DEV void kerr_rhs_vjp_hand(double M, double a, double r, double th, const double w[4],
                              const double kb[4], double* Xr, double* Xth, double W[4],
                              double* ga) {
  double s, c;
  ::sincos(th, &s, &c);
  // ---- forward: the geometry's base quantities and its fields ----
  const double r2 = r * r, a2 = a * a, s2 = s * s, c2 = c * c, sc = s * c;
  const double sig = r2 + a2 * c2;
  const double del = (r - 2.0 * M) * r + a2;
  const double rho = r2 + a2;
  const double sd = sig * del;
  const double R = 1.0 / (sd * s2);
  const double iSD = s2 * R, iS = del * iSD, iD = sig * iSD, is2 = sd * R;
  const double iS2 = iS * iS, iD2 = iD * iD;
  const double sm2r = a2 * c2 - r2;
  const double X3 = a2 * (r * s2 + M * c2) - M * r2;
  const double Y8 = sig + rho;
  const double BA = rho * rho - a2 * del * s2;
  const double Z13 = del - a2 * s2;
  const double dtt_r = 2.0 * M * sm2r * iS2;
  const double dtt_th = 4.0 * M * r * a2 * sc * iS2;
  const double drr_r = 2.0 * X3 * iD2;
  const double drr_th = -2.0 * a2 * sc * iD;
  const double dthth_r = 2.0 * r;
  const double dthth_th = -2.0 * a2 * sc;
  const double dphph_r = 2.0 * r * s2 + 2.0 * M * a2 * (s2 * s2) * sm2r * iS2;
  const double dphph_th = 2.0 * rho * sc + 4.0 * M * r * a2 * sc * s2 * Y8 * iS2;
  const double dtph_r = -2.0 * M * a * s2 * sm2r * iS2;
  const double dtph_th = -4.0 * M * r * a * sc * rho * iS2;
  const double gtt = -BA * iSD;
  const double gtph = -2.0 * M * r * a * iSD;
  const double gphph = Z13 * iSD * is2;
  const double hrr = -0.5 * del * iS;
  const double hthth = -0.5 * iS;
  // ---- forward: the contraction's intermediates ----
  const double vt = w[0], vr = w[1], vth = w[2], vph = w[3];
  const double A1 = dtt_r * vt + dtph_r * vph, A2 = dtt_th * vt + dtph_th * vph;
  const double B1 = dtph_r * vt + dphph_r * vph, B2 = dtph_th * vt + dphph_th * vph;
  const double Et = vr * A1 + vth * A2, Ep = vr * B1 + vth * B2;
  const double vt2 = vt * vt, vr2 = vr * vr, vth2 = vth * vth, vph2 = vph * vph;
  const double two_tp = 2.0 * vt * vph, two_rt = 2.0 * vr * vth;
  const double S1 = drr_r * vr2 - dtt_r * vt2 - dthth_r * vth2 - dphph_r * vph2 +
                    drr_th * two_rt - dtph_r * two_tp;
  const double S2 = dthth_th * vth2 - dtt_th * vt2 - drr_th * vr2 - dphph_th * vph2 +
                    dthth_r * two_rt - dtph_th * two_tp;
  // ---- reverse through the contraction ----
  // acc0 = -(gtt Et + gtph Ep), acc3 = -(gtph Et + gphph Ep)
  const double gttb = -kb[0] * Et;
  const double gtphb = -kb[0] * Ep - kb[3] * Et;
  const double gphphb = -kb[3] * Ep;
  const double Etb = -kb[0] * gtt - kb[3] * gtph;
  const double Epb = -kb[0] * gtph - kb[3] * gphph;
  // acc1 = hrr S1, acc2 = hthth S2
  const double hrrb = kb[1] * S1, hththb = kb[2] * S2;
  const double S1b = kb[1] * hrr, S2b = kb[2] * hthth;
  // Et = vr A1 + vth A2, Ep = vr B1 + vth B2
  const double A1b = Etb * vr, A2b = Etb * vth, B1b = Epb * vr, B2b = Epb * vth;
  double vtb = A1b * dtt_r + A2b * dtt_th + B1b * dtph_r + B2b * dtph_th;
  double vrb = Etb * A1 + Epb * B1;
  double vthb = Etb * A2 + Epb * B2;
  double vphb = A1b * dtph_r + A2b * dtph_th + B1b * dphph_r + B2b * dphph_th;
  // the fields' cotangents (through the energy sums and the two quadratic rows)
  const double dtt_rb = A1b * vt - S1b * vt2;
  const double dtph_rb = A1b * vph + B1b * vt - S1b * two_tp;
  const double dphph_rb = B1b * vph - S1b * vph2;
  const double drr_rb = S1b * vr2;
  const double dthth_rb = -S1b * vth2 + S2b * two_rt;
  const double drr_thb = S1b * two_rt - S2b * vr2;
  const double dtt_thb = A2b * vt - S2b * vt2;
  const double dtph_thb = A2b * vph + B2b * vt - S2b * two_tp;
  const double dphph_thb = B2b * vph - S2b * vph2;
  const double dthth_thb = S2b * vth2;
  // the quadratic rows' velocity cotangents
  const double vt2b = -S1b * dtt_r - S2b * dtt_th;
  const double vr2b = S1b * drr_r - S2b * drr_th;
  const double vth2b = -S1b * dthth_r + S2b * dthth_th;
  const double vph2b = -S1b * dphph_r - S2b * dphph_th;
  const double two_tpb = -S1b * dtph_r - S2b * dtph_th;
  const double two_rtb = S1b * drr_th + S2b * dthth_r;
  vtb += 2.0 * (vt * vt2b + vph * two_tpb);
  vphb += 2.0 * (vph * vph2b + vt * two_tpb);
  vrb += 2.0 * (vr * vr2b + vth * two_rtb);
  vthb += 2.0 * (vth * vth2b + vr * two_rtb);
  W[0] += vtb;
  W[1] += vrb;
  W[2] += vthb;
  W[3] += vphb;
  // ---- reverse through the geometry ----
  double rb = 0.0, ab = 0.0, a2b = 0.0, s2b = 0.0, c2b = 0.0, scb = 0.0, sigb = 0.0,
         delb = 0.0, rhob = 0.0, iSb = 0.0, iDb = 0.0, is2b = 0.0, sm2rb = 0.0, r2b = 0.0;
  {  // dtt_r = 2 M sm2r iS^2
    sm2rb += dtt_rb * 2.0 * M * iS2;
    iSb += dtt_rb * 4.0 * M * sm2r * iS;
  }
  {  // dtt_th = 4 M r a2 sc iS^2
    const double k = dtt_thb * 4.0 * M;
    rb += k * a2 * sc * iS2;
    a2b += k * r * sc * iS2;
    scb += k * r * a2 * iS2;
    iSb += k * r * a2 * sc * 2.0 * iS;
  }
  {  // drr_r = 2 X3 iD^2, X3 = a2 (r s2 + M c2) - M r2
    const double xb = drr_rb * 2.0 * iD2;
    iDb += drr_rb * 4.0 * X3 * iD;
    a2b += xb * (r * s2 + M * c2);
    rb += xb * a2 * s2;
    s2b += xb * a2 * r;
    c2b += xb * a2 * M;
    r2b -= xb * M;
  }
  {  // drr_th = -2 a2 sc iD
    const double k = -2.0 * drr_thb;
    a2b += k * sc * iD;
    scb += k * a2 * iD;
    iDb += k * a2 * sc;
  }
  rb += 2.0 * dthth_rb;            // dthth_r = 2 r
  a2b += -2.0 * dthth_thb * sc;    // dthth_th = -2 a2 sc
  scb += -2.0 * dthth_thb * a2;
  {  // dphph_r = 2 r s2 + 2 M a2 s2^2 sm2r iS^2
    rb += 2.0 * dphph_rb * s2;
    s2b += 2.0 * dphph_rb * r;
    const double k = dphph_rb * 2.0 * M;
    a2b += k * (s2 * s2) * sm2r * iS2;
    s2b += k * a2 * 2.0 * s2 * sm2r * iS2;
    sm2rb += k * a2 * (s2 * s2) * iS2;
    iSb += k * a2 * (s2 * s2) * sm2r * 2.0 * iS;
  }
  {  // dphph_th = 2 rho sc + 4 M r a2 sc s2 Y8 iS^2, Y8 = sig + rho
    rhob += 2.0 * dphph_thb * sc;
    scb += 2.0 * dphph_thb * rho;
    const double k = dphph_thb * 4.0 * M;
    rb += k * a2 * sc * s2 * Y8 * iS2;
    a2b += k * r * sc * s2 * Y8 * iS2;
    scb += k * r * a2 * s2 * Y8 * iS2;
    s2b += k * r * a2 * sc * Y8 * iS2;
    const double yb = k * r * a2 * sc * s2 * iS2;
    sigb += yb;
    rhob += yb;
    iSb += k * r * a2 * sc * s2 * Y8 * 2.0 * iS;
  }
  {  // dtph_r = -2 M a s2 sm2r iS^2
    const double k = -2.0 * M * dtph_rb;
    ab += k * s2 * sm2r * iS2;
    s2b += k * a * sm2r * iS2;
    sm2rb += k * a * s2 * iS2;
    iSb += k * a * s2 * sm2r * 2.0 * iS;
  }
  {  // dtph_th = -4 M r a sc rho iS^2
    const double k = -4.0 * M * dtph_thb;
    rb += k * a * sc * rho * iS2;
    ab += k * r * sc * rho * iS2;
    scb += k * r * a * rho * iS2;
    rhob += k * r * a * sc * iS2;
    iSb += k * r * a * sc * rho * 2.0 * iS;
  }
  {  // gtt = -BA iS iD, BA = rho^2 - a2 del s2
    const double bab = -gttb * iSD;
    iSb += -gttb * BA * iD;
    iDb += -gttb * BA * iS;
    rhob += bab * 2.0 * rho;
    a2b += -bab * del * s2;
    delb += -bab * a2 * s2;
    s2b += -bab * a2 * del;
  }
  {  // gtph = -2 M r a iS iD
    const double k = -2.0 * M * gtphb;
    rb += k * a * iSD;
    ab += k * r * iSD;
    iSb += k * r * a * iD;
    iDb += k * r * a * iS;
  }
  {  // gphph = Z13 iS iD is2, Z13 = del - a2 s2
    const double zb = gphphb * iSD * is2;
    iSb += gphphb * Z13 * iD * is2;
    iDb += gphphb * Z13 * iS * is2;
    is2b += gphphb * Z13 * iSD;
    delb += zb;
    a2b -= zb * s2;
    s2b -= zb * a2;
  }
  delb += -0.5 * hrrb * iS;  // hrr = -del iS / 2
  iSb += -0.5 * hrrb * del;
  iSb += -0.5 * hththb;      // hthth = -iS / 2
  // the base quantities
  a2b += sm2rb * c2;  // sm2r = a2 c2 - r2
  c2b += sm2rb * a2;
  r2b -= sm2rb;
  sigb -= iSb * iS2;         // iS = 1 / sig
  delb -= iDb * iD2;         // iD = 1 / del
  s2b -= is2b * is2 * is2;   // is2 = 1 / s2
  r2b += sigb;               // sig = r2 + a2 c2
  a2b += sigb * c2;
  c2b += sigb * a2;
  rb += delb * (2.0 * r - 2.0 * M);  // del = r^2 - 2 M r + a2
  a2b += delb;
  r2b += rhob;               // rho = r2 + a2
  a2b += rhob;
  rb += 2.0 * r * r2b;
  ab += 2.0 * a * a2b;
  const double sb = 2.0 * s * s2b + c * scb, cb = 2.0 * c * c2b + s * scb;
  *Xr += rb;
  *Xth += sb * c - cb * s;
  *ga += ab;
}

}  // namespace gg
