// Trilinear hexahedra (nshl = 8): the NS+VOF quench and temperature
// element routines (src/solveQuenching.f90:122-882) with the 2x2x2 rule
// (src/genGP_GW.f90:355-389) and linhexshl (src/eval_shape_FEM.f90:148-196),
// assembled like the tets: an element pass writes per-Gauss-point records
// and the element's residual rows, a row pass (one warp per CSR row) expands
// the blocks of A's row and adds them in ascending element id.  Unlike a
// linear tet, a hex has different gradients at every Gauss point, so the
// row pass sums each block over the 8 points.  Included into assemble.cu's
// anonymous namespace (it uses its helpers).

// node signs of linhexshl: N_a = (1 + sx xi)(1 + sy eta)(1 + sz zeta) / 8
__constant__ signed char c_hex_sign[8][3] = {{-1, 1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, 1, 1},
                                             {-1, -1, -1}, {1, -1, -1}, {1, -1, 1}, {-1, -1, 1}};
// 2x2x2 points (genGPandGW, weights 1)
__device__ __forceinline__ void hex_gp(int g, double& xi, double& eta, double& ze) {
  const double q = 0.57735026918963;
  xi = (g & 1) ? q : -q;
  eta = (g & 2) ? q : -q;
  ze = (g & 4) ? q : -q;
}
template <typename T>
__device__ __forceinline__ T hex_N(int g, int a) {
  double xi, eta, ze;
  hex_gp(g, xi, eta, ze);
  return (T)((1.0 + c_hex_sign[a][0] * xi) * (1.0 + c_hex_sign[a][1] * eta) * (1.0 + c_hex_sign[a][2] * ze) * 0.125);
}

template <int KIND> struct HexLay;
//   NS+VOF record per point: g(8x3) w KA KB MM KDP dphi(3) uadv(3) rho rt
//   tauLS src eps ufac plfac pad(2); then the residual rows 8x5
template <> struct HexLay<OVS_ASM_NSVOF> {
  static constexpr int GPW = 44, RHS0 = 8 * 44, NF = 5, SW = 8 * 44 + 40, NV = 24;
};
//   T record per point: g(8x3) w HK uadv(3) rcp dSe trc; then 8 residuals
template <> struct HexLay<OVS_ASM_TEM> {
  static constexpr int GPW = 32, RHS0 = 8 * 32, NF = 1, SW = 8 * 32 + 8, NV = 1;
};

//   NS+VOF record per point for the tensor-core path: dxi/dx (3x3, row k =
//   xi_k) w KA KB MM KDP dphi(3) v(3) = dxi/dx uadv, rho rt tauLS src eps
//   ufac plfac pad; then the residual rows 8x5
struct HexTcLay {
  static constexpr int GPW = 28, RHS0 = 8 * 28, SW = 8 * 28 + 40;
};

// eval_shape_fem for a hex at point g on x+d: global gradients, DetJ, G
template <typename T>
__device__ __forceinline__ T hex_geometry(int gp, const T r[8][16], const T lo[8][4], T g[8][3], T G[3][3],
                                          T (*Aio)[3] = nullptr) {
  double xi, eta, ze;
  hex_gp(gp, xi, eta, ze);
  T dN[8][3];
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    const double sx = c_hex_sign[a][0], sy = c_hex_sign[a][1], sz = c_hex_sign[a][2];
    dN[a][0] = (T)(sx * (1.0 + sy * eta) * (1.0 + sz * ze) * 0.125);
    dN[a][1] = (T)(sy * (1.0 + sx * xi) * (1.0 + sz * ze) * 0.125);
    dN[a][2] = (T)(sz * (1.0 + sx * xi) * (1.0 + sy * eta) * 0.125);
  }
  // dx/dxi from coordinates relative to node 0 (sum_a dN_a = 0), so the
  // FP32 path keeps the edge lengths to full precision
  T A[3][3], Ai[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T s = 0;
#pragma unroll
      for (int a = 1; a < 8; ++a) s += ((r[a][i] - r[0][i]) + (lo[a][i] - lo[0][i])) * dN[a][j];
      A[i][j] = s;
    }
  Ai[0][0] = A[1][1] * A[2][2] - A[2][1] * A[1][2];
  Ai[0][1] = A[2][1] * A[0][2] - A[0][1] * A[2][2];
  Ai[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
  T tmp = (T)1.0 / (Ai[0][0] * A[0][0] + Ai[0][1] * A[1][0] + Ai[0][2] * A[2][0]);
  Ai[0][0] *= tmp; Ai[0][1] *= tmp; Ai[0][2] *= tmp;
  Ai[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * tmp;
  Ai[1][1] = (A[0][0] * A[2][2] - A[2][0] * A[0][2]) * tmp;
  Ai[1][2] = (A[1][0] * A[0][2] - A[0][0] * A[1][2]) * tmp;
  Ai[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * tmp;
  Ai[2][1] = (A[2][0] * A[0][1] - A[0][0] * A[2][1]) * tmp;
  Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * tmp;
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int j = 0; j < 3; ++j) g[a][j] = dN[a][0] * Ai[0][j] + dN[a][1] * Ai[1][j] + dN[a][2] * Ai[2][j];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) G[i][j] = Ai[0][i] * Ai[0][j] + Ai[1][i] * Ai[1][j] + Ai[2][i] * Ai[2][j];
  if (Aio)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Aio[i][j] = Ai[i][j];
  return (T)1.0 / tmp;
}

template <typename T>
__device__ __forceinline__ typename Wide<T>::type hex_phi(const T r[8][16], const T lo[8][4], int k, int gp) {
  using W = typename Wide<T>::type;
  W s = 0.0;
#pragma unroll
  for (int a = 0; a < 8; ++a) s += ((W)r[a][k] + (W)lo[a][3]) * hex_N<double>(gp, a);
  return s;
}

template <typename T>
__device__ __forceinline__ void store_n(T* dst, const T* v, int n) {
  for (int k = 0; k < n; ++k) dst[k] = v[k];
}

// element pass, NS+VOF quench on a hex (src/solveQuenching.f90:295-523);
// TC: write the compact records of the tensor-core matrix pass instead
template <typename T, bool TC = false>
__device__ void hex_summarize_nsvof(const ovs_params& p, const T r[8][16], const T lo[8][4], bool fluid,
                                    T* out, double& tamax, int& nbad) {
  using W = typename Wide<T>::type;
  using L = HexLay<OVS_ASM_NSVOF>;
  constexpr int RHS0 = TC ? HexTcLay::RHS0 : L::RHS0;
  const T fact2 = (T)(p.alfi * p.delt * p.gami);
  const T taut = (T)(4.0 / (p.delt * p.delt));
  const T rhoa = (T)p.rhoa, rhow = (T)p.rhow, ts = (T)p.ts;
  // reciprocals of the launch constants, taken once: the point formulas
  // multiply by them where the reference divides (as the tet routines)
  const T its = (T)(1.0 / p.ts), irhoa = (T)(1.0 / p.rhoa), irhow = (T)(1.0 / p.rhow);
  const T ira = irhoa - irhow;
  const bool kdc_on = fabs(p.ns_kdc_w) + fabs(p.ns_kdc_a) > 0.0;
  const bool kdcphi_on = fabs(p.lsc_kdc) > 0.0;
  T ru[8][3], rp[8], rf[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) { ru[n][0] = ru[n][1] = ru[n][2] = 0; rp[n] = 0; rf[n] = 0; }
  for (int gp = 0; gp < 8; ++gp) {
    T g[8][3], G[3][3], Ai[3][3];
    const T detj = hex_geometry<T>(gp, r, lo, g, G, Ai);
    if (!(detj > (T)0)) nbad = 1;
    const T w = detj;   // hex weights are 1
    T GG = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) GG += G[i][j] * G[i][j];
    const T trG = G[0][0] + G[1][1] + G[2][2];
    T N[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) N[a] = hex_N<T>(gp, a);
    T du[3][3], dp[3], dphi[3], ui[3], umi[3], aci[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      ui[i] = umi[i] = aci[i] = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j) du[i][j] = 0;
      dp[i] = dphi[i] = 0;
    }
    T pri = 0, rphii = 0, Ti = 0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        ui[i] += r[a][3 + i] * N[a];
        umi[i] += r[a][6 + i] * N[a];
        aci[i] += r[a][9 + i] * N[a];
#pragma unroll
        for (int j = 0; j < 3; ++j) du[i][j] += r[a][3 + i] * g[a][j];
        dp[i] += r[a][12] * g[a][i];
        dphi[i] += r[a][13] * g[a][i];
      }
      pri += r[a][12] * N[a];
      rphii += r[a][14] * N[a];
      Ti += r[a][15] * N[a];
    }
    const T divu = du[0][0] + du[1][1] + du[2][2];
    const W phid = hex_phi<T>(r, lo, 13, gp);
    const T phii = (T)phid;
    const W phicd = clamp01(phid);
    const T phic = (T)phicd;
    T mdot, dmd;
    if (Ti > ts) {
      mdot = (T)p.c_evap * (T)(1.0 - phicd) * rhow * (Ti - ts) * its;
      dmd = -(T)p.c_evap * rhow * (Ti - ts) * its * (T)p.c_dmdot;
    } else {
      mdot = (T)p.c_cond * phic * rhoa * (Ti - ts) * its;
      dmd = (T)p.c_cond * rhoa * (Ti - ts) * its * (T)p.c_dmdot;
    }
    const T vdot = mdot * irhoa - mdot * irhow;
    T rho, mu;
    if (fluid) {
      rho = (T)(p.rhow * (1.0 - phicd) + p.rhoa * phicd);
      mu = (T)(p.muw * (1.0 - phicd) + p.mua * phicd);
    } else {
      rho = (T)p.rhos; mu = (T)p.mus;
    }
    const T lambda = (T)(-2.0 / 3.0) * mu;
    if (phid < 0.0 || phid > 1.0) dmd = 0;
    const T uadv[3] = {ui[0] - umi[0], ui[1] - umi[1], ui[2] - umi[2]};
    T tmp1[3], rL[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const T conv = du[i][0] * uadv[0] + du[i][1] * uadv[1] + du[i][2] * uadv[2];
      tmp1[i] = rho * aci[i] + rho * conv - (T)p.gravvec[i] * rho;
      rL[i] = tmp1[i] + dp[i];
    }
    const T res_phi = rphii + (uadv[0] * dphi[0] + uadv[1] * dphi[1] + uadv[2] * dphi[2]) + phii * vdot - mdot * irhoa;
    const T taua = quad_uGu<T>(uadv, G);
    const T irho = (T)1.0 / rho;
    const T nu = mu * irho;
    const T taud = nu * nu * (T)12.0 * GG;
    const T tauM = irho * inv_sqrt(taut + taua + taud);
    const T tauLS = inv_sqrt(taut + taua);
    const T tauC = rho * sqrt(taua + taud) / trG;
    if ((double)taua > tamax) tamax = (double)taua;   // CFL number: delt sqrt(max taua), in the kernel
    T kdc = 0;
    if (kdc_on) {
      const double nk = (double)(p.ns_kdc_w * (1.0 - phicd) + p.ns_kdc_a * phicd);
      const T rr = rL[0] * rL[0] + rL[1] * rL[1] + rL[2] * rL[2];
      kdc = (T)low_word(nk) * sqrt(rr / GG);
    }
    T kdphi = 0;
    if (kdcphi_on) kdphi = (T)p.lsc_kdc * fabs(res_phi) / sqrt(GG);
    const T mupk = mu + kdc;
    const T dmdi = dmd * ira;
    const T wf = fluid ? w : (T)0;   // solid elements contribute nothing
    if constexpr (TC) {
      T rec[HexTcLay::GPW];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j) rec[3 * k + j] = Ai[k][j];
      rec[9] = wf;
      rec[10] = fluid ? fact2 * mupk * w : (T)0;
      rec[11] = fluid ? fact2 * (tauC + lambda) * w : (T)0;
      rec[12] = fluid ? fact2 * w * tauM : (T)0;
      rec[13] = fluid ? fact2 * w * kdphi : (T)0;
      rec[14] = dphi[0]; rec[15] = dphi[1]; rec[16] = dphi[2];
#pragma unroll
      for (int k = 0; k < 3; ++k) rec[17 + k] = Ai[k][0] * uadv[0] + Ai[k][1] * uadv[1] + Ai[k][2] * uadv[2];
      rec[20] = rho; rec[21] = rho * tauM; rec[22] = tauLS;
      rec[23] = vdot + phii * ira * dmd - dmd * irhoa;
      rec[24] = fact2 * wf * tauC * dmdi * dmdi;
      rec[25] = fact2 * tauC * dmdi * wf;
      rec[26] = fact2 * dmdi * wf;
      rec[27] = 0;
      store_n(out + gp * HexTcLay::GPW, rec, HexTcLay::GPW);
    } else {
      T rec[L::GPW];
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) rec[3 * a + d] = g[a][d];
      rec[24] = wf;
      rec[25] = fluid ? fact2 * mupk * w : (T)0;
      rec[26] = fluid ? fact2 * (tauC + lambda) * w : (T)0;
      rec[27] = fluid ? fact2 * w * tauM : (T)0;
      rec[28] = fluid ? fact2 * w * kdphi : (T)0;
      rec[29] = dphi[0]; rec[30] = dphi[1]; rec[31] = dphi[2];
      rec[32] = uadv[0]; rec[33] = uadv[1]; rec[34] = uadv[2];
      rec[35] = rho; rec[36] = rho * tauM; rec[37] = tauLS;
      rec[38] = vdot + phii * ira * dmd - dmd * irhoa;
      rec[39] = fact2 * wf * tauC * dmdi * dmdi;
      rec[40] = fact2 * tauC * dmdi * wf;
      rec[41] = fact2 * dmdi * wf;
      rec[42] = 0; rec[43] = 0;
      store_n(out + gp * L::GPW, rec, L::GPW);
    }
    if (!fluid) continue;
    T svis[8], gdphi[8], c[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      T sv = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k)
        sv += g[n][0] * (du[0][k] + du[k][0]) + g[n][1] * (du[1][k] + du[k][1]) + g[n][2] * (du[2][k] + du[k][2]);
      svis[n] = sv;
      gdphi[n] = g[n][0] * dphi[0] + g[n][1] * dphi[1] + g[n][2] * dphi[2];
      c[n] = uadv[0] * g[n][0] + uadv[1] * g[n][1] + uadv[2] * g[n][2];
    }
    const T tdiv = -pri + tauC * divu;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
        ru[n][i] += w * (-N[n] * tmp1[i] - g[n][i] * tdiv + g[n][i] * tauC * vdot - g[n][i] * lambda * divu -
                         mupk * svis[n] + rho * c[n] * (-tauM * rL[i]));
      rp[n] += w * (-N[n] * (divu - vdot) + (g[n][0] * rL[0] + g[n][1] * rL[1] + g[n][2] * rL[2]) * (-tauM));
      rf[n] += w * (-(N[n] + tauLS * c[n]) * res_phi - kdphi * gdphi[n] + N[n] * dmdi * tauC * (divu - vdot));
    }
  }
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    T* orh = out + RHS0 + 5 * n;
    orh[0] = ru[n][0]; orh[1] = ru[n][1]; orh[2] = ru[n][2]; orh[3] = rp[n]; orh[4] = rf[n];
  }
}

// element pass, temperature on a hex (src/solveQuenching.f90:712-856);
// record layout of this pass: xd(0:2) u(3:5) um(6:8) phi(9) T(10) rT(11)
template <typename T>
__device__ void hex_summarize_tem(const ovs_params& p, const T r[8][16], const T lo[8][4], bool fluid, T* out,
                                  double& tamax, int& nbad) {
  using W = typename Wide<T>::type;
  using L = HexLay<OVS_ASM_TEM>;
  const T fact2 = (T)(p.alfi * p.gami * p.delt);
  const T ts = (T)p.ts, cpw = (T)p.cpw, cpa = (T)p.cpa, lh = (T)p.lh;
  const T its = (T)(1.0 / p.ts), itref = (T)(1.0 / p.tref), taut = (T)(4.0 / (p.delt * p.delt));
  const bool kdc_on = fabs(p.tem_kdc) > 0.0;
  T rt[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) rt[n] = 0;
  for (int gp = 0; gp < 8; ++gp) {
    T g[8][3], G[3][3];
    const T detj = hex_geometry<T>(gp, r, lo, g, G);
    if (!(detj > (T)0)) nbad = 1;
    const T w = detj;
    T GG = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) GG += G[i][j] * G[i][j];
    T N[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) N[a] = hex_N<T>(gp, a);
    T dT[3] = {0, 0, 0}, ui[3] = {0, 0, 0}, umi[3] = {0, 0, 0};
    T Ti = 0, rTi = 0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        dT[j] += r[a][10] * g[a][j];
        ui[j] += r[a][3 + j] * N[a];
        umi[j] += r[a][6 + j] * N[a];
      }
      Ti += r[a][10] * N[a];
      rTi += r[a][11] * N[a];
    }
    T gdT[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) gdT[n] = g[n][0] * dT[0] + g[n][1] * dT[1] + g[n][2] * dT[2];
    const W phid = hex_phi<T>(r, lo, 9, gp);
    const W phicd = clamp01(phid);
    const T phic = (T)phicd;
    T mdot, dmdT;
    if (Ti > ts) {
      mdot = (T)p.c_evap * (T)(1.0 - phicd) * (T)p.rhow * (Ti - ts) * its;
      dmdT = (T)p.c_evap * (T)(1.0 - phicd) * (T)p.rhow * its * (T)p.c_dmdot;
    } else {
      mdot = (T)p.c_cond * phic * (T)p.rhoa * (Ti - ts) * its;
      dmdT = (T)p.c_cond * phic * (T)p.rhoa * its * (T)p.c_dmdot;
    }
    T rho, cp, hk, rcp;
    if (fluid) {
      rho = (T)(p.rhow * (1.0 - phicd) + p.rhoa * phicd);
      cp = (T)(p.cpw * (1.0 - phicd) + p.cpa * phicd);
      hk = (T)(p.kappaw * (1.0 - phicd) + p.kappaa * phicd);
      rcp = (T)((p.rhow * p.cpw) * (1.0 - phicd) + (p.rhoa * p.cpa) * phicd);
    } else {
      rho = (T)p.rhos; cp = (T)p.cps; hk = (T)p.kappas; rcp = (T)(p.rhos * p.cps);
    }
    const T uadv[3] = {ui[0] - umi[0], ui[1] - umi[1], ui[2] - umi[2]};
    const T Se = ((cpw - cpa) * (Ti - ts) - lh) * mdot;
    const T udT = uadv[0] * dT[0] + uadv[1] * dT[1] + uadv[2] * dT[2];
    const T res = rcp * (rTi + udT) - Se;
    const T taua = quad_uGu<T>(uadv, G);
    T tt = taua + taut;
    const T ircp = (T)1.0 / (rho * cp);
    const T kk = hk * ircp;
    tt = tt + kk * kk * (T)12.0 * GG;
    const T tauT = ircp * inv_sqrt(tt);
    if ((double)taua > tamax) tamax = (double)taua;   // CFL number: delt sqrt(max taua), in the kernel
    T kdcT = 0;
    if (kdc_on && fluid) kdcT = (T)p.tem_kdc * fabs(res) * inv_sqrt(GG) * itref;
    const T dSe = (cpw - cpa) * mdot + ((cpw - cpa) * (Ti - ts) - lh) * dmdT;
    T rec[L::GPW];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int d = 0; d < 3; ++d) rec[3 * a + d] = g[a][d];
    rec[24] = w;
    rec[29] = rcp;
    if (fluid) {
      rec[25] = fact2 * (hk + kdcT) * w;
      rec[26] = uadv[0]; rec[27] = uadv[1]; rec[28] = uadv[2];
      rec[30] = dSe; rec[31] = tauT * rcp;
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        const T cn = uadv[0] * g[n][0] + uadv[1] * g[n][1] + uadv[2] * g[n][2];
        rt[n] += w * (-N[n] * rcp * (rTi + udT) + N[n] * Se - rcp * tauT * cn * res - (hk + kdcT) * gdT[n]);
      }
    } else {
      rec[25] = fact2 * hk * w;
      rec[26] = rec[27] = rec[28] = 0; rec[30] = 0; rec[31] = 0;
#pragma unroll
      for (int n = 0; n < 8; ++n) rt[n] += w * (-N[n] * rcp * rTi - hk * gdT[n]);
    }
    store_n(out + gp * L::GPW, rec, L::GPW);
  }
#pragma unroll
  for (int n = 0; n < 8; ++n) out[L::RHS0 + n] = rt[n];
}

template <typename T, int KIND, bool TC = false>
__global__ void __launch_bounds__(64) hex_element_kernel(const SumArgs a) {
  using L = HexLay<KIND>;
  constexpr int SW = TC ? HexTcLay::SW : L::SW;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  double tamax = 0.0;   // the element's largest taua over its points
  int nbad = 0;
  if (e < a.E) {
    T r[8][16], lo[8][4];
    const T* rec = reinterpret_cast<const T*>(a.rec);
#pragma unroll
    for (int n = 0; n < 8; ++n) load_rec(rec, a.ien[8 * (size_t)e + n], r[n], lo[n]);
    const bool fluid = __ldg(a.elm_id + e) == a.p.fluid_elm_id;
    T* out = reinterpret_cast<T*>(a.sum) + (size_t)e * SW;
    if constexpr (KIND == OVS_ASM_NSVOF) hex_summarize_nsvof<T, TC>(a.p, r, lo, fluid, out, tamax, nbad);
    else hex_summarize_tem<T>(a.p, r, lo, fluid, out, tamax, nbad);
  }
  double cfl = (double)a.p.delt * sqrt(tamax);   // as the tet element pass
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    cfl = fmax(cfl, __shfl_xor_sync(0xffffffffu, cfl, off));
    nbad += __shfl_xor_sync(0xffffffffu, nbad, off);
  }
  if ((threadIdx.x & 31) == 0) {
    cfl_max(a.cfl_bits, cfl);
    if (nbad) atomicAdd(a.flags, nbad);
  }
}

// Block (row node la, column node b) of a hex from its records: the
// per-point forms of the tet block sums (see expand_block), summed over the
// 8 points.
template <typename T, int KIND>
__device__ __forceinline__ void hex_expand_block(const ovs_params& p, const T* sm, int la, int b, T* o, T* rv) {
  using L = HexLay<KIND>;
  if constexpr (KIND == OVS_ASM_TEM) {
    const T fact1 = (T)p.almi, fact2 = (T)(p.alfi * p.gami * p.delt);
    T X = 0;
    for (int gp = 0; gp < 8; ++gp) {
      const T* q = sm + gp * L::GPW;
      const T ga[3] = {q[3 * la], q[3 * la + 1], q[3 * la + 2]};
      const T gb[3] = {q[3 * b], q[3 * b + 1], q[3 * b + 2]};
      const T w = q[24], HK = q[25], rcp = q[29], dSe = q[30], trc = q[31];
      const T uadv[3] = {q[26], q[27], q[28]};
      const T Na = hex_N<T>(gp, la), Nb = hex_N<T>(gp, b);
      const T ca = ga[0] * uadv[0] + ga[1] * uadv[1] + ga[2] * uadv[2];
      const T cb = gb[0] * uadv[0] + gb[1] * uadv[1] + gb[2] * uadv[2];
      const T aw = w * (Na + trc * ca);
      X += aw * (rcp * (fact1 * Nb + fact2 * cb) - fact2 * dSe * Nb) + HK * (ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2]);
    }
    o[0] = X;
    rv[0] = sm[L::RHS0 + la];
  } else {
    const T fact1 = (T)p.almi, fact2 = (T)(p.alfi * p.delt * p.gami);
#pragma unroll
    for (int v = 0; v < 24; ++v) o[v] = 0;
    for (int gp = 0; gp < 8; ++gp) {
      const T* q = sm + gp * L::GPW;
      const T ga[3] = {q[3 * la], q[3 * la + 1], q[3 * la + 2]};
      const T gb[3] = {q[3 * b], q[3 * b + 1], q[3 * b + 2]};
      T s[20];
#pragma unroll
      for (int k = 0; k < 20; k += 4) ldv4(q + 24 + k, s + k);
      const T w = s[0], KA = s[1], KB = s[2], MM = s[3], KDP = s[4];
      const T dphi[3] = {s[5], s[6], s[7]}, uadv[3] = {s[8], s[9], s[10]};
      const T rho = s[11], rt = s[12], tls = s[13], src = s[14], eps = s[15], ufac = s[16], plfac = s[17];
      const T Na = hex_N<T>(gp, la), Nb = hex_N<T>(gp, b);
      const T ca = uadv[0] * ga[0] + uadv[1] * ga[1] + uadv[2] * ga[2];
      const T cb = uadv[0] * gb[0] + uadv[1] * gb[1] + uadv[2] * gb[2];
      const T gab = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
      const T beta = fact1 * Nb + fact2 * cb;
      const T S = w * rho * (Na + rt * ca) * beta;
      const T P = fact2 * w * Nb, Q = fact2 * w * rt * ca, R = fact2 * w * Na, Tt = w * rt * beta;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) o[4 * i + j] += KA * ga[j] * gb[i] + KB * ga[i] * gb[j] + (i == j ? KA * gab + S : (T)0);
        o[4 * i + 3] += -ga[i] * P + gb[i] * Q;
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) o[12 + d] += gb[d] * R + ga[d] * Tt;
      o[15] += MM * gab;
      const T gam = w * (Na + tls * ca);
#pragma unroll
      for (int d = 0; d < 3; ++d) o[16 + d] += dphi[d] * (fact2 * gam * Nb) - gb[d] * (ufac * Na);
      o[19] += gam * (beta + fact2 * Nb * src) + KDP * gab + eps * Na * Nb;
#pragma unroll
      for (int d = 0; d < 3; ++d) o[20 + d] += ga[d] * (ufac * Nb);
      o[23] += -plfac * Na * Nb;
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) rv[f] = sm[L::RHS0 + 5 * la + f];
  }
}

// ------------------------------------------------------------------------
// Tensor-core element matrices (FP32 NS+VOF hexahedra).
//
// Every block value t of the quench matrix is, per Gauss point g, a bilinear
// form in the features (N, grad N) of the row node a and the column node b.
// Written with the reference-element features f_g = (N, dN/dxi) (the same
// for every element), the element's block is
//     K_t[a][b] = sum_g sum_{r,s} C'_{t,g}[r][s] f_g[r][a] f_g[s][b],
// with C' = T^T C T, T = diag(1, dxi/dx^T) mapping reference to physical
// gradients.  So all element matrices of a tile are ONE dense product
//     D[(t, e), (a, b)] = A[(t, e), (g, r, s)] * W[(g, r, s), (a, b)],
// M = 8 types x 16 elements = 128, K = 8 points x 16 = 128, N = 64, with
// the constant W = f_g (x) f_g shared by all elements, on tcgen05 (kind::tf32,
// A and W K-major in shared memory without swizzle, D in TMEM).  FP32
// accuracy comes from the 3xTF32 split A_hi W_hi + A_hi W_lo + A_lo W_hi
// (W's split precomputed on the host).  One CTA of 128 threads per SM loops
// over tiles of 16 elements with 256 threads; thread (element el, point g)
// of each half builds its point's 4x4 C' for 4 of a group's 8 slot values
// (three groups of 8 cover the 24; the value is a template parameter),
// thread 0 issues the 48 MMAs of a group into its 64 TMEM columns and
// commits them to an mbarrier; the epilogue reads the 192 columns back and
// writes each element's 64 x 24 block values (slot order) through shared
// memory with coalesced stores.

constexpr int TC_EB = 16;                                 // elements per tile
constexpr int TC_KST = 64 * 24 + 4;                       // staging floats per element (padded)
constexpr int TC_A_BYTES = 128 * 128 * 4;                 // one A operand (hi or lo)
constexpr int TC_W_BYTES = 64 * 128 * 4;                  // one W operand (hi or lo)
constexpr int TC_SMEM = 2 * TC_A_BYTES + 2 * TC_W_BYTES;  // 192 KB
constexpr int TC_TMEM_COLS = 256;                         // 3 groups x 64 columns
constexpr long TC_WAIT_LIMIT = 1L << 26;                  // bounded mbarrier wait (iterations)

struct HexTcArgs {
  const float* rec;    // element records, HexTcLay
  const float* w;      // W hi then W lo, canonical K-major no-swizzle layout (2 x 8192 floats)
  float* kbuf;         // E x 64 x 24 block values
  int* flags;          // [2] set when an mbarrier wait gave up
  int E;
  float fact1, fact2;
};

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ float tc_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
// shared-memory matrix descriptor: SWIZZLE_NONE, K-major, version 1
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t dcol, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
               ::"r"(dcol), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
  uint32_t done = 0;
  for (long it = 0; it < TC_WAIT_LIMIT && !done; ++it)
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(done) : "r"(bar), "r"(parity) : "memory");
  return done != 0;
}
__device__ __forceinline__ void tc_ld16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// C' (reference features, row-major 4x4: [r][s], r on the row node a) of slot
// value t at one point, from the point record q (HexTcLay): the per-point
// forms of hex_expand_block with u.grad N = v . dN/dxi (v = dxi/dx uadv),
// grad N_a . grad N_b = dN_a/dxi Gh dN_b/dxi (Gh = dxi/dx dxi/dx^T) and the
// physical derivative j = dN/dxi . a_j (a_j column j of dxi/dx).
template <int t>
__device__ __forceinline__ void tc_coeffs(const float* q, const float Gh[3][3], float f1, float f2, float C[16]) {
#pragma unroll
  for (int k = 0; k < 16; ++k) C[k] = 0.f;
  const float w = q[9], KA = q[10], KB = q[11], MM = q[12], KDP = q[13];
  const float v[3] = {q[17], q[18], q[19]};
  const float rho = q[20], rt = q[21], tls = q[22], src = q[23], eps = q[24], ufac = q[25], plfac = q[26];
  auto A = [&](int k, int j) { return q[3 * k + j]; };   // dxi_k/dx_j
  if constexpr (t < 12 && (t & 3) != 3) {  // K(i, j)
    constexpr int i = t >> 2, j = t & 3;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) C[4 * (1 + k) + 1 + l] = KA * A(k, j) * A(l, i) + KB * A(k, i) * A(l, j);
    if constexpr (i == j) {
      const float al[4] = {1.f, rt * v[0], rt * v[1], rt * v[2]};
      const float be[4] = {f1, f2 * v[0], f2 * v[1], f2 * v[2]};
      const float wr = w * rho;
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) C[4 * r + c] += wr * al[r] * be[c];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l) C[4 * (1 + k) + 1 + l] += KA * Gh[k][l];
    }
  } else if constexpr (t < 12) {           // G(i)
    constexpr int i = t >> 2;
    const float fw = f2 * w;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      C[4 * (1 + k)] = -fw * A(k, i);
#pragma unroll
      for (int l = 0; l < 3; ++l) C[4 * (1 + k) + 1 + l] = fw * rt * v[k] * A(l, i);
    }
  } else if constexpr (t < 15) {           // D(d)
    constexpr int d = t - 12;
    const float wrt = w * rt;
#pragma unroll
    for (int l = 0; l < 3; ++l) C[1 + l] = f2 * w * A(l, d);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      C[4 * (1 + k)] = wrt * A(k, d) * f1;
#pragma unroll
      for (int l = 0; l < 3; ++l) C[4 * (1 + k) + 1 + l] = wrt * A(k, d) * f2 * v[l];
    }
  } else if constexpr (t == 15) {          // M
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) C[4 * (1 + k) + 1 + l] = MM * Gh[k][l];
  } else if constexpr (t < 19) {           // LSU(d)
    constexpr int d = t - 16;
    const float c0 = q[14 + d] * f2 * w;
    C[0] = c0;
#pragma unroll
    for (int k = 0; k < 3; ++k) C[4 * (1 + k)] = c0 * tls * v[k];
#pragma unroll
    for (int l = 0; l < 3; ++l) C[1 + l] = -ufac * A(l, d);
  } else if constexpr (t == 19) {          // LS
    const float al[4] = {1.f, tls * v[0], tls * v[1], tls * v[2]};
    const float ga[4] = {f1 + f2 * src, f2 * v[0], f2 * v[1], f2 * v[2]};
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) C[4 * r + c] = w * al[r] * ga[c];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) C[4 * (1 + k) + 1 + l] += KDP * Gh[k][l];
    C[0] += eps;
  } else if constexpr (t < 23) {           // ULS(d)
    constexpr int d = t - 20;
#pragma unroll
    for (int k = 0; k < 3; ++k) C[4 * (1 + k)] = ufac * A(k, d);
  } else {                                 // PLS
    C[0] = -plfac;
  }
}

// A rows m = 16 t8 + el, 16-byte chunk kc = 4 g + r (hi and lo operands)
template <int t>
__device__ __forceinline__ void tc_store_type(const float* q, const float Gh[3][3], float f1, float f2,
                                              unsigned char* sAh, unsigned char* sAl, int el, int g) {
  float C[16];
  tc_coeffs<t>(q, Gh, f1, f2, C);
  const int m = 16 * (t & 7) + el;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int off = (4 * g + r) * 2048 + (m >> 3) * 128 + (m & 7) * 16;
    float4 h, l;
    h.x = tc_tf32(C[4 * r]); h.y = tc_tf32(C[4 * r + 1]); h.z = tc_tf32(C[4 * r + 2]); h.w = tc_tf32(C[4 * r + 3]);
    l.x = tc_tf32(C[4 * r] - h.x); l.y = tc_tf32(C[4 * r + 1] - h.y);
    l.z = tc_tf32(C[4 * r + 2] - h.z); l.w = tc_tf32(C[4 * r + 3] - h.w);
    *reinterpret_cast<float4*>(sAh + off) = h;
    *reinterpret_cast<float4*>(sAl + off) = l;
  }
}

// the 8 slot values of group GRP: the warp-uniform half hf of the CTA builds 4 of them
template <int GRP>
__device__ __forceinline__ void tc_store_group(int hf, const float* q, const float Gh[3][3], float f1, float f2,
                                               unsigned char* sAh, unsigned char* sAl, int el, int g) {
  if (hf == 0) {
    tc_store_type<8 * GRP + 0>(q, Gh, f1, f2, sAh, sAl, el, g);
    tc_store_type<8 * GRP + 1>(q, Gh, f1, f2, sAh, sAl, el, g);
    tc_store_type<8 * GRP + 2>(q, Gh, f1, f2, sAh, sAl, el, g);
    tc_store_type<8 * GRP + 3>(q, Gh, f1, f2, sAh, sAl, el, g);
  } else {
    tc_store_type<8 * GRP + 4>(q, Gh, f1, f2, sAh, sAl, el, g);
    tc_store_type<8 * GRP + 5>(q, Gh, f1, f2, sAh, sAl, el, g);
    tc_store_type<8 * GRP + 6>(q, Gh, f1, f2, sAh, sAl, el, g);
    tc_store_type<8 * GRP + 7>(q, Gh, f1, f2, sAh, sAl, el, g);
  }
}

constexpr int TC_THREADS = 256;

// builds group GRP's operands, issues its MMAs and waits for them; false when the wait gave up
template <int GRP>
__device__ __forceinline__ bool tc_group(int hf, const float* q, const float Gh[3][3], float f1, float f2,
                                         unsigned char* sAh, unsigned char* sAl, unsigned char* sWh,
                                         unsigned char* sWl, int el, int g, uint32_t tm, uint32_t barp,
                                         uint32_t idesc, uint32_t& phase) {
  tc_store_group<GRP>(hf, q, Gh, f1, f2, sAh, sAl, el, g);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (threadIdx.x == 0) {
    const uint32_t dcol = tm + 64 * GRP;
    const uint32_t ah = tc_smem(sAh), al = tc_smem(sAl), wh = tc_smem(sWh), wl = tc_smem(sWl);
    for (int ks = 0; ks < 16; ++ks)
      tc_mma(dcol, tc_desc(ah + ks * 4096, 2048, 128), tc_desc(wh + ks * 2048, 1024, 128), idesc, ks > 0);
    for (int ks = 0; ks < 16; ++ks)
      tc_mma(dcol, tc_desc(ah + ks * 4096, 2048, 128), tc_desc(wl + ks * 2048, 1024, 128), idesc, 1u);
    for (int ks = 0; ks < 16; ++ks)
      tc_mma(dcol, tc_desc(al + ks * 4096, 2048, 128), tc_desc(wh + ks * 2048, 1024, 128), idesc, 1u);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(barp)
                 : "memory");
  }
  // the operands are free again (and, after the last group, D is complete)
  const bool done = tc_wait(barp, phase);
  const bool ok = __syncthreads_and(done) != 0;
  if (ok) phase ^= 1u;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return ok;
}

__global__ void __launch_bounds__(TC_THREADS, 1) hex_tc_matrix_kernel(const HexTcArgs a) {
  extern __shared__ __align__(1024) unsigned char tc_sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tbase;
  unsigned char* sAh = tc_sm;
  unsigned char* sAl = tc_sm + TC_A_BYTES;
  unsigned char* sWh = tc_sm + 2 * TC_A_BYTES;
  unsigned char* sWl = sWh + TC_W_BYTES;
  float* kst = reinterpret_cast<float*>(tc_sm);             // epilogue staging over the A operands
  const int t = threadIdx.x, wid = t >> 5, lane = t & 31;
  const int hf = t >> 7, tt = t & 127;                      // half of the CTA (4 of each group's 8 values)
  const int el = tt & 15, g = tt >> 4;                      // this thread's element and point
  {  // W hi / lo into shared memory (already in the canonical layout)
    const float4* src = reinterpret_cast<const float4*>(a.w);
    float4* dst = reinterpret_cast<float4*>(sWh);
    for (int i = t; i < 2 * TC_W_BYTES / 16; i += TC_THREADS) dst[i] = src[i];
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (wid == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&tbase)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tbase, barp = tc_smem(&bar);
  // kind::tf32, F32 accumulate, A and B K-major, N = 64, M = 128
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
  const float f1 = a.fact1, f2 = a.fact2;
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (a.E + TC_EB - 1) / TC_EB;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * TC_EB, e = e0 + el;
    float q[HexTcLay::GPW];
    if (e < a.E) {
      const float4* r4 = reinterpret_cast<const float4*>(a.rec + (size_t)e * HexTcLay::SW + g * HexTcLay::GPW);
#pragma unroll
      for (int k = 0; k < HexTcLay::GPW / 4; ++k) {
        const float4 x = __ldg(r4 + k);
        q[4 * k] = x.x; q[4 * k + 1] = x.y; q[4 * k + 2] = x.z; q[4 * k + 3] = x.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < HexTcLay::GPW; ++k) q[k] = 0.f;
    }
    float Gh[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l) Gh[k][l] = q[3 * k] * q[3 * l] + q[3 * k + 1] * q[3 * l + 1] + q[3 * k + 2] * q[3 * l + 2];
    ok = tc_group<0>(hf, q, Gh, f1, f2, sAh, sAl, sWh, sWl, el, g, tm, barp, idesc, phase) &&
         tc_group<1>(hf, q, Gh, f1, f2, sAh, sAl, sWh, sWl, el, g, tm, barp, idesc, phase) &&
         tc_group<2>(hf, q, Gh, f1, f2, sAh, sAl, sWh, sWl, el, g, tm, barp, idesc, phase);
    if (!ok) break;
    // epilogue: warp quartet hf reads columns [32 hf, 32 hf + 32) of each group's 64, lanes 32 (wid % 4) + lane
    {
      const int w4 = wid & 3, m = 32 * w4 + lane, t8 = m >> 4, eli = m & 15;
      float* dst = kst + eli * TC_KST;
#pragma unroll
      for (int grp = 0; grp < 3; ++grp)
#pragma unroll
        for (int c = 0; c < 32; c += 16) {
          const int c0 = 32 * hf + c;
          float v[16];
          tc_ld16(tm + ((uint32_t)(32 * w4) << 16) + 64 * grp + c0, v);
#pragma unroll
          for (int j = 0; j < 16; ++j) dst[(c0 + j) * 24 + 8 * grp + t8] = v[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    {
      const int nel = min(TC_EB, a.E - e0);
      float4* out = reinterpret_cast<float4*>(a.kbuf + (size_t)e0 * 1536);
      for (int i = t; i < nel * 384; i += TC_THREADS) {
        const int ee = i / 384, j4 = i - ee * 384;
        out[i] = *reinterpret_cast<const float4*>(kst + ee * TC_KST + 4 * j4);
      }
    }
    __syncthreads();   // staging (the A operands) free for the next tile
  }
  if (!ok) {   // give the MMAs in flight one more bounded wait before TMEM is released
    tc_wait(barp, phase);
    if (t == 0) atomicOr(a.flags + 2, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (wid == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TC_TMEM_COLS));
}

// shared memory per warp: blocks [4 elements][8 columns][BSTR], RHS rows
// [4][RSTR], row accumulator [max_deg][NVP]; ints: slots [4][8], columns
template <typename T, int KIND> struct HexSmem {
  static constexpr int NV = HexLay<KIND>::NV, NF = HexLay<KIND>::NF;
  static constexpr int CH = 4;
  static constexpr int NVP = (NV < 4) ? 1 : NV;
  static constexpr int BSTR = (NV < 4) ? 1 : NV + 16 / (int)sizeof(T);
  static constexpr int RSTR = NF + 1;
  __host__ __device__ static size_t bytes(int max_deg) {
    size_t b = sizeof(T) * ((size_t)8 * CH * BSTR + (size_t)CH * RSTR + (size_t)max_deg * NVP);
    b = (b + 15) & ~(size_t)15;
    b += sizeof(int) * ((size_t)8 * CH + max_deg);
    return (b + 15) & ~(size_t)15;
  }
};

template <typename T, int KIND, bool TC = false>
__global__ void __launch_bounds__(128) hex_rows_kernel(const AsmArgs a) {
  using S = HexSmem<T, KIND>;
  using L = HexLay<KIND>;
  constexpr int NV = S::NV, NF = S::NF, NVP = S::NVP, BSTR = S::BSTR, RSTR = S::RSTR, CH = S::CH;
  constexpr int WARPS = 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned masks[24];
  if (threadIdx.x < 24) masks[threadIdx.x] = (KIND == OVS_ASM_TEM) ? (TB | (TB << 8) | (TB << 16)) : mask_of(threadIdx.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* base = smem_raw + (size_t)wid * S::bytes(a.max_deg);
  T* blk = reinterpret_cast<T*>(base);                 // [CH][8][BSTR]
  T* rvs = blk + 8 * CH * BSTR;                        // [CH][RSTR]
  T* acc = rvs + CH * RSTR;                            // [max_deg][NVP]
  size_t off = sizeof(T) * ((size_t)8 * CH * BSTR + (size_t)CH * RSTR + (size_t)a.max_deg * NVP);
  off = (off + 15) & ~(size_t)15;
  int* slot = reinterpret_cast<int*>(base + off);      // [CH][8]
  int* cols = slot + 8 * CH;                           // [max_deg]
  const T* sum = reinterpret_cast<const T*>(a.rec);
  const uint2* n2s8 = reinterpret_cast<const uint2*>(a.n2s);
  const int jl = lane >> 3, bl = lane & 7;
  for (int A = blockIdx.x * WARPS + wid; A < a.N; A += gridDim.x * WARPS) {
    const int rp = a.rowptr[A], deg = a.rowptr[A + 1] - rp;
    const int ep = a.n2e_ptr[A], ne = a.n2e_ptr[A + 1] - ep;
    for (int s = lane; s < deg; s += 32) cols[s] = a.colidx[rp + s];
    for (int q = lane; q < deg * NVP; q += 32) acc[q] = (T)0;
    T racc = (T)0;
    __syncwarp();
    for (int c0 = 0; c0 < ne; c0 += CH) {
      const int nc = min(CH, ne - c0);
      if (jl < nc) {
        const int packed = __ldg(a.n2e + ep + c0 + jl);
        const uint2 sl = __ldg(n2s8 + ep + c0 + jl);
        const int e = packed >> 3, la = packed & 7;
        T o[NVP], rv[NF];
        if constexpr (TC) {   // block values of the tensor-core pass, slot order
          const float4* kb = reinterpret_cast<const float4*>(reinterpret_cast<const float*>(a.kbuf) +
                                                             ((size_t)e * 64 + la * 8 + bl) * 24);
#pragma unroll
          for (int v = 0; v < 6; ++v) {
            const float4 x = __ldg(kb + v);
            o[4 * v] = x.x; o[4 * v + 1] = x.y; o[4 * v + 2] = x.z; o[4 * v + 3] = x.w;
          }
#pragma unroll
          for (int f = 0; f < NF; ++f) rv[f] = sum[(size_t)e * HexTcLay::SW + HexTcLay::RHS0 + 5 * la + f];
        } else {
          hex_expand_block<T, KIND>(a.p, sum + (size_t)e * L::SW, la, bl, o, rv);
        }
        T* dst = blk + (jl * 8 + bl) * BSTR;
        if constexpr (NV >= 4) {
#pragma unroll
          for (int v = 0; v < NV; v += 4) store_row<4>(dst + v, o + v);
        } else {
          dst[0] = o[0];
        }
        const unsigned word = bl < 4 ? sl.x : sl.y;
        slot[jl * 8 + bl] = (int)((word >> (8 * (bl & 3))) & 0xffu);
        if (bl == 0) {
#pragma unroll
          for (int f = 0; f < NF; ++f) rvs[jl * RSTR + f] = rv[f];
        }
      }
      __syncwarp();
      // ordered reduction: the 8 blocks of one element go to distinct slots
      if constexpr (NV >= 4) {
        constexpr int NG = NV / 4;
        for (int j = 0; j < nc; ++j) {
          for (int q = lane; q < 8 * NG; q += 32) {
            const int b = q / NG, gidx = q - b * NG;
            Vec4<T>::add(acc + slot[j * 8 + b] * NVP + gidx * 4, blk + (j * 8 + b) * BSTR + gidx * 4);
          }
          __syncwarp();
        }
      } else {
        for (int j = 0; j < nc; ++j) {
          if (lane < 8) acc[slot[j * 8 + lane]] += blk[j * 8 + lane];
          __syncwarp();
        }
      }
      if (lane < NF)
        for (int j = 0; j < nc; ++j) racc += rvs[j * RSTR + lane];
      __syncwarp();
    }
    // row write with the Dirichlet treatment (as for the tets)
    const unsigned ibA = a.ibc[A];
    if (a.mat) {
      T* outp = reinterpret_cast<T*>(a.vals) + (size_t)rp * NV;
      const T cnt = (T)ne;
      if constexpr (NV >= 4) {
        constexpr int NG = NV / 4;
        for (int q = lane; q < deg * NG; q += 32) {
          const int s = q / NG, gidx = q - s * NG;
          const int B = cols[s];
          const unsigned ibB = __ldg(a.ibc + B);
          const bool dg = B == A;
          T v4[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const unsigned m = masks[4 * gidx + t];
            T val = acc[s * NVP + 4 * gidx + t];
            if ((ibA & m & 0xffu) || ((ibB << 8) & m & 0xff00u)) val = (T)0;
            if (dg && ((ibA << 16) & m & 0xff0000u)) val = cnt;
            v4[t] = val;
          }
          store_row<4>(outp + (size_t)s * NV + 4 * gidx, v4);
        }
      } else {
        for (int q = lane; q < deg; q += 32) {
          const int B = cols[q];
          const unsigned ibB = __ldg(a.ibc + B);
          T val = acc[q];
          if ((ibA & TB) || (ibB & TB)) val = (T)0;
          if (B == A && (ibA & TB)) val = cnt;
          outp[q] = val;
        }
      }
    }
    if (a.vec && lane < NF) {
      unsigned bit;
      if (KIND == OVS_ASM_TEM) bit = TB;
      else bit = (lane < 3) ? (1u << lane) : (lane == 3 ? PB : FB);
      T v = (ibA & bit) ? (T)0 : racc;
      if (!isfinite((double)v)) atomicOr(a.flags + 1, 1);
      reinterpret_cast<T*>(a.rhs)[(size_t)lane * a.N + A] = v;
    }
    __syncwarp();
  }
}

template <typename T, int KIND>
int launch_assemble_hex(ovs_ctx* c, const AsmArgs& a0, const SumArgs& sa, int parts) {
  constexpr bool can_tc = std::is_same<T, float>::value && KIND == OVS_ASM_NSVOF;
  const bool tc = can_tc && c->hex_tc;
  AsmArgs a = a0;
  if (tc) {
    int st;
    if ((st = hex_tc_prepare(c))) return st;
    a.kbuf = c->hex_kbuf;
  }
  if (parts & 1) {
    if (tc) {
      if constexpr (can_tc) {
        hex_element_kernel<T, KIND, true><<<(sa.E + 63) / 64, 64, 0, c->stream>>>(sa);
        ++c->launches;
        OVS_CUDA_TRY(cudaGetLastError());
        HexTcArgs ta;
        ta.rec = reinterpret_cast<const float*>(sa.sum);
        ta.w = c->hex_w;
        ta.kbuf = reinterpret_cast<float*>(c->hex_kbuf);
        ta.flags = c->flags;
        ta.E = sa.E;
        ta.fact1 = (float)sa.p.almi;
        ta.fact2 = (float)(sa.p.alfi * sa.p.delt * sa.p.gami);
        OVS_CUDA_TRY(cudaFuncSetAttribute(hex_tc_matrix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
        const int ntiles = (sa.E + TC_EB - 1) / TC_EB;
        const int grid = ntiles < c->num_sms ? ntiles : c->num_sms;
        if (grid > 0) {
          hex_tc_matrix_kernel<<<grid, TC_THREADS, TC_SMEM, c->stream>>>(ta);
          ++c->launches;
          OVS_CUDA_TRY(cudaGetLastError());
        }
      }
    } else {
      hex_element_kernel<T, KIND><<<(sa.E + 63) / 64, 64, 0, c->stream>>>(sa);
      ++c->launches;
      OVS_CUDA_TRY(cudaGetLastError());
    }
  }
  if (!(parts & 2)) return OVS_OK;
  using S = HexSmem<T, KIND>;
  const size_t smem = S::bytes(a.max_deg) * 4;
  auto kern = tc ? hex_rows_kernel<T, KIND, can_tc> : hex_rows_kernel<T, KIND, false>;
  OVS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  OVS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem));
  if (per_sm < 1) return OVS_ERR_ARG;
  long need = ((long)c->N + 3) / 4;
  long grid = (long)per_sm * c->num_sms * 4;
  if (grid > need) grid = need;
  if (grid < 1) grid = 1;
  kern<<<(int)grid, 128, smem, c->stream>>>(a);
  ++c->launches;
  OVS_CUDA_TRY(cudaGetLastError());
  return OVS_OK;
}
