// Coefficient table of the tau-banded preconditioner P = P_tau (x) I_Vs.
//
// The values are the hand-built table of the reference
// (preconditioners_orig/precon_manual.py:36-166), kept identical because the
// preconditioner is part of the reference's algorithm: for each tau-distance
// r = 0..6 the values of the first rows ("edge"), the bulk value ("middle")
// and the values of the last rows ("tail") of that band, and the wrap-around
// corner values at (0, Nt-r) / (Nt-r, 0) for r = 1..5.  The reference stores
// them as complex64, so they are float here.  Band 6 starts at row 1, the
// others at row 0; the table is defined for Nt >= 26.
#pragma once

namespace qedf {

constexpr int PRE_NBAND = 7;
constexpr int PRE_MIN_LTAU = 26;
#define QEDF_PRE_LAYOUT                                                     \
  {10, 12, 8, 8, 9, 11, 7}, /* edge lengths */                              \
      {9, 8, 7, 6, 8, 10, 7}, /* tail lengths */                            \
      {0, 10, 22, 30, 38, 47, 58}, /* edge offsets */                       \
      {0, 9, 17, 24, 30, 38, 48}, /* tail offsets */                        \
      {0, 0, 0, 0, 0, 0, 1} /* first row of each band */

#define QEDF_PRE_EDGE_VALUES                                                                  \
  {0.91698223f, 1.02107012f, 1.1740706f,  1.24646831f, 1.28092396f, 1.29741096f, 1.30534041f, \
   1.30917168f, 1.3110323f,  1.31193936f, /* r = 1 */ 0.475227f, 0.69804072f, 0.80315554f,    \
   0.85303694f, 0.87684089f, 0.88826168f, 0.89376724f, 0.89643389f, 0.89773124f, 0.89836514f, \
   0.89867532f, 0.89882821f, /* r = 2 */ 0.32525402f, 0.47824016f, 0.550632f, 0.58508581f,    \
   0.60157132f, 0.60949975f, 0.61333305f, 0.61519265f, /* r = 3 */ 0.22288805f, 0.32804558f,  \
   0.3779504f,  0.40176818f, 0.41319385f, 0.4187026f,  0.42137364f, 0.42267111f,              \
   /* r = 4 */ 0.15300766f, 0.22541766f, 0.25988016f, 0.27637246f, 0.28430402f, 0.28813654f, \
   0.29000109f, 0.29090756f, 0.291352f, /* r = 5 */ 0.10518534f, 0.15511395f, 0.17894313f,    \
   0.190377f,   0.19588688f, 0.1985613f,  0.19986567f, 0.20050026f, 0.20081173f, 0.20096488f, \
   0.20104057f, /* r = 6 */ 0.10691644f, 0.12341493f, 0.13135427f, 0.13519259f, 0.13706173f,  \
   0.13796897f, 0.13841458f}

#define QEDF_PRE_TAIL_VALUES                                                                  \
  {1.31167626f, 1.31074941f, 1.30885756f, 1.30498219f, 1.29699361f, 1.28042281f, 1.24588311f, \
   1.17343438f, 1.02052784f, /* r = 1 */ 0.89785033f, 0.89652652f, 0.89382064f, 0.88826007f,  \
   0.87676316f, 0.85285789f, 0.80287397f, 0.69771057f, /* r = 2 */ 0.61507541f, 0.61318511f,  \
   0.60930747f, 0.60131705f, 0.58475631f, 0.5502165f,  0.47778079f, /* r = 3 */ 0.42132217f,  \
   0.41861743f, 0.41305307f, 0.40155935f, 0.37766892f, 0.3276957f, /* r = 4 */ 0.29132634f,   \
   0.29086968f, 0.28994057f, 0.28805143f, 0.28417516f, 0.27618375f, 0.25962788f, 0.22511749f, \
   /* r = 5 */ 0.20103745f, 0.20095888f, 0.20079921f, 0.20047785f, 0.19982809f, 0.19850214f, \
   0.19579838f, 0.19023941f, 0.17874525f, 0.15486649f, /* r = 6 */ 0.13839549f, 0.13793865f,  \
   0.13701266f, 0.13511762f, 0.13124515f, 0.12326149f, 0.10670882f}

#define QEDF_PRE_MIDDLE_VALUES \
  {1.312381281f, 0.8989771f, 0.616974f, 0.42391914f, 0.29178312f, 0.20111492f, 0.13884714f}

#define QEDF_PRE_CORNER_VALUES {-0.47505581f, -0.32495788f, -0.22264314f, -0.15278356f, -0.10501137f}

// value of entry k (0-based from the band's first row) of band r with n entries
struct PreTable {
  int edge_len[PRE_NBAND];
  int tail_len[PRE_NBAND];
  int edge_off[PRE_NBAND];
  int tail_off[PRE_NBAND];
  int start[PRE_NBAND];
  float edge[65];
  float tail[55];
  float middle[PRE_NBAND];
  float corner[5];
};

template <typename T>
__host__ __device__ inline float pre_band_value(const T& tab, int r, int k, int n) {
  if (k < tab.edge_len[r]) return tab.edge[tab.edge_off[r] + k];
  const int tail0 = n - tab.tail_len[r];
  if (k >= tail0) return tab.tail[tab.tail_off[r] + (k - tail0)];
  return tab.middle[r];
}

// Calls fn(col, value) for every nonzero of row t of P_tau (Nt >= 26).
template <typename T, typename Fn>
__host__ __device__ inline void pre_row(const T& tab, int Nt, int t, Fn fn) {
  fn(t, pre_band_value(tab, 0, t, Nt));
  for (int r = 1; r < PRE_NBAND; ++r) {
    const int s = tab.start[r];
    const int n = Nt - r - s;
    if (t - r >= s) fn(t - r, pre_band_value(tab, r, t - r - s, n));
    if (t >= s && t + r < Nt) fn(t + r, pre_band_value(tab, r, t - s, n));
  }
  for (int r = 1; r <= 5; ++r) {
    if (t == 0) fn(Nt - r, tab.corner[r - 1]);
    if (t == Nt - r) fn(0, tab.corner[r - 1]);
  }
}

}  // namespace qedf
