// Host-side element tables for libvoxfea (double precision, computed once per
// solver):
//   KE(nu)   24x24 unit-cube hex8 stiffness at E = 1, 2x2x2 Gauss quadrature,
//            J = 0.5 I  -- the reference's _hex8_KE (core/fea.py:31-76)
//   K_lam, K_mu  with KE(E, nu) = lam*K_lam + mu*K_mu (per-voxel Poisson ratio)
//   B0       6x24 centroid strain-displacement matrix (core/fea.py:79-122)
//   Galerkin child tables G[ch] = P_ch^T K P_ch: a fine voxel at child position
//            ch of a coarse voxel, seen from the coarse voxel's 24 DOFs through
//            the trilinear prolongation (core/multigrid.py:42-73).
#pragma once

namespace vf {

// Reference local corner offsets (core/fea.py:33-36).
static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

inline void hex8_B(double xi, double eta, double zeta, double B[6][24]) {
  for (int r = 0; r < 6; ++r)
    for (int j = 0; j < 24; ++j) B[r][j] = 0.0;
  for (int i = 0; i < 8; ++i) {
    const double a = 2 * kCorner[i][0] - 1, b = 2 * kCorner[i][1] - 1, c = 2 * kCorner[i][2] - 1;
    // dN/dxi / J with J = 0.5 I
    const double bx = a * (1 + b * eta) * (1 + c * zeta) / 8.0 / 0.5;
    const double by = b * (1 + a * xi) * (1 + c * zeta) / 8.0 / 0.5;
    const double bz = c * (1 + a * xi) * (1 + b * eta) / 8.0 / 0.5;
    const int c0 = 3 * i;
    B[0][c0] = bx;
    B[1][c0 + 1] = by;
    B[2][c0 + 2] = bz;
    B[3][c0] = by;
    B[3][c0 + 1] = bx;
    B[4][c0 + 1] = bz;
    B[4][c0 + 2] = by;
    B[5][c0] = bz;
    B[5][c0 + 2] = bx;
  }
}

inline void hex8_integrate(const double C[6][6], double K[576]) {
  for (int i = 0; i < 576; ++i) K[i] = 0.0;
  const double g = 1.0 / 1.7320508075688772;   // 1/sqrt(3)
  const double gp[2] = {-g, g};
  double B[6][24], CB[6][24];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        hex8_B(gp[a], gp[b], gp[c], B);
        for (int r = 0; r < 6; ++r)
          for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += C[r][k] * B[k][j];
            CB[r][j] = s;
          }
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += B[k][i] * CB[k][j];
            K[i * 24 + j] += s * 0.125;
          }
      }
}

// tab = [KE(nu) | K_lam | K_mu]
inline void hex8_tables(double nu, double tab[1728], double B0[144]) {
  double C[6][6] = {};
  const double c = 1.0 / ((1 + nu) * (1 - 2 * nu));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) C[i][j] = c * (i == j ? 1 - nu : nu);
  for (int i = 3; i < 6; ++i) C[i][i] = c * (1 - 2 * nu) / 2;
  hex8_integrate(C, tab);
  double CL[6][6] = {}, CM[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) CL[i][j] = 1.0;
  for (int i = 0; i < 3; ++i) CM[i][i] = 2.0;
  for (int i = 3; i < 6; ++i) CM[i][i] = 1.0;
  hex8_integrate(CL, tab + 576);
  hex8_integrate(CM, tab + 1152);
  double B[6][24];
  hex8_B(0.0, 0.0, 0.0, B);
  for (int r = 0; r < 6; ++r)
    for (int j = 0; j < 24; ++j) B0[r * 24 + j] = B[r][j];
}

inline double w1d(int d) { return d == 0 ? 1.0 : ((d == 1 || d == -1) ? 0.5 : 0.0); }

// G[ch] (8 x 576) = P_ch^T K P_ch for one 24x24 K.
inline void galerkin_child_tables(const double* K, double* G) {
  for (int ch = 0; ch < 8; ++ch) {
    const int ci = ch & 1, cj = (ch >> 1) & 1, ck = ch >> 2;
    double W[8][8];   // W[i][a]: weight of coarse corner a at the child's node i
    for (int i = 0; i < 8; ++i)
      for (int a = 0; a < 8; ++a) {
        const int fx = ci + kCorner[i][0], fy = cj + kCorner[i][1], fz = ck + kCorner[i][2];
        W[i][a] = w1d(fx - 2 * kCorner[a][0]) * w1d(fy - 2 * kCorner[a][1]) * w1d(fz - 2 * kCorner[a][2]);
      }
    double* Gc = G + ch * 576;
    for (int a = 0; a < 8; ++a)
      for (int r = 0; r < 3; ++r)
        for (int b = 0; b < 8; ++b)
          for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int i = 0; i < 8; ++i) {
              if (W[i][a] == 0.0) continue;
              for (int j = 0; j < 8; ++j) s += W[i][a] * W[j][b] * K[(3 * i + r) * 24 + 3 * j + c];
            }
            Gc[(3 * a + r) * 24 + 3 * b + c] = s;
          }
  }
}

}  // namespace vf
