// CPU oracle for the RUMD Lennard-Jones / Nose-Hoover NVT time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is a CPU restatement of the reference
// algorithm, used by tests/, by __graft_entry__.smoke() and by the
// cpu_baseline / --impl reference legs of bench.py as the checker and as the
// timed CPU baseline.  It is never linked into, or called by, the product
// library (rumd_b200/).
//
// Parity anchors (reference paths are relative to the RUMD source tree):
//   * Pot_LJ_12_6::SetParams            include/rumd/PairPotential.h:202-207
//   * Pot_IPL_12_6::ComputeInteraction  include/rumd/PairPotential.h:161-168
//   * Pot_LJ_12_6_smooth_2_4            include/rumd/PairPotential.h:218-256
//   * Pot_IPL_n                         include/rumd/PairPotential.h:603-637
//   * fij (NS/SP/SF cut-off handling)   include/rumd/PairPotential.h:1198-1244
//   * shift constants p10/p11           src/PairPotential.cu:82-125
//   * calculateDistance / wrap          include/rumd/SimulationBox.h:111-155
//   * cell grid, cell coordinates       src/NeighborList.cu:717-732, 1106-1140
//   * stable key sort (thrust)          include/rumd/Sample.h:174-188
//   * sorted cell scan (order, skin)    src/NeighborList.cu:1204-1319
//   * displacement trigger              src/NeighborList.cu:970-997
//   * list capacity estimate            src/NeighborList.cu:595-606
//   * Nose-Hoover leap-frog             src/IntegratorNVT.cu:364-418
//   * thermostat update                 src/IntegratorNVT.cu:82-92, 426-437
//   * momentum zeroing                  src/IntegratorNVT.cu:176-183, 444-471
//   * leap-frog kinetic energy          src/IntegratorNVT.cu:316-356
//   * host FP64 sums (pe, virial)       src/Sample.cu:353-391
//   * degrees of freedom 3N-3           src/Sample.cu:301
//
// FP64 mode (orc_md_run_f64) restates the reference built after
// changeToDouble.sh (changeToDouble.sh:1-189): every quantity is a double,
// including the shift constants s(rc) rc, u(rc) (from rc, A12, A6 of the
// table) and omega^2 = 4 pi^2 / tau^2.
//
// Arithmetic: compiled with -ffp-contract=off so that every float operation
// rounds exactly where it is written.  Where the reference's device build
// contracts a product and a sum into one fused multiply-add, the restatement
// writes fmaf() explicitly (see dist2_ref / cell_coord_ref); those forms are
// the ones the GPU kernels reproduce bit for bit, and a GPU test checks that
// nvcc's default contraction of the reference expressions yields the same bits.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API extern "C" __attribute__((visibility("default")))

enum { ORC_NS = 0, ORC_SP = 1, ORC_SF = 2 };
static const int NP = 12;  // NumParam, include/rumd/rumd_base.h

// ---------------------------------------------------------------------------
// Parameter table (reference layout: params[(ti*T + tj)*12 + k])
// ---------------------------------------------------------------------------

// Pot_IPL_12_6::ComputeInteraction, host float arithmetic (no contraction).
static float ipl_12_6_f32(float dist2, const float* p, float* u_acc) {
  float invDist2 = 1.0f / dist2;
  float invDist6 = invDist2 * invDist2 * invDist2;
  float temp = p[1] * invDist6;
  float s = invDist6 * invDist2 * (12.f * temp + 6.f * p[2]);
  *u_acc += invDist6 * (temp + p[2]);
  return s;
}

// PairPotential::CopyParamsToGPU for one (i,j) row (src/PairPotential.cu:82-125):
// p11 = u(rc), p10 = s(rc) rc from the float pair function, then the row is
// stored at (i,j) and mirrored to (j,i) (assume_Newton3 defaults to true,
// src/PairPotential.cu:55).
static void store_row(int ntypes, float* params, int i, int j, float* row,
                      float (*pair)(float, const float*, float*)) {
  float u = 0.f, s = 0.f;
  float Rcut = row[0];
  if (Rcut > 0.0f) s = pair(Rcut * Rcut, row, &u);
  row[NP - 1] = u;
  row[NP - 2] = s * Rcut;
  std::memcpy(&params[(i * ntypes + j) * NP], row, NP * sizeof(float));
  if (i != j) std::memcpy(&params[(j * ntypes + i) * NP], row, NP * sizeof(float));
}

// Pot_LJ_12_6::SetParams + PairPotential::CopyParamsToGPU for one (i,j) pair,
// mirrored to (j,i) (assume_Newton3 defaults to true, src/PairPotential.cu:55).
ORC_API void orc_lj_set_params(int ntypes, float* params, int i, int j,
                               float sigma, float epsilon, float rcut) {
  float row[NP];
  std::memset(row, 0, sizeof(row));
  row[0] = rcut * sigma;
  row[1] = (float)(4. * epsilon * std::pow((double)sigma, 12.));
  row[2] = (float)(-4. * epsilon * std::pow((double)sigma, 6.));
  store_row(ntypes, params, i, j, row, ipl_12_6_f32);
}

// Pot_LJ_12_6_smooth_2_4::ComputeInteraction, host float arithmetic
// (include/rumd/PairPotential.h:248-255).
static float smooth_2_4_f32(float dist2, const float* p, float* u_acc) {
  float Dist2 = dist2 * p[1];
  float invDist2 = 1.0f / Dist2;
  float invDist6 = invDist2 * invDist2 * invDist2;
  float s = p[2] * p[1] * (invDist2 * invDist6 * (12.f * invDist6 - 6.f) - 2.0f * p[3] - 4.0f * p[4] * Dist2);
  *u_acc += p[2] * (invDist6 * (invDist6 - 1.0f) + p[3] * Dist2 + p[4] * Dist2 * Dist2);
  return s;
}

// Pot_IPL_n::ComputeInteraction, host float arithmetic
// (include/rumd/PairPotential.h:630-636).
static float ipl_n_f32(float dist2, const float* p, float* u_acc) {
  float invDist2 = 1.0f / (dist2 * p[1]);
  float invDist_n = expf(logf(invDist2) * p[3] * 0.5f);
  float s = p[1] * p[2] * p[3] * invDist_n * invDist2;
  *u_acc += p[2] * invDist_n;
  return s;
}

// Pot_LJ_12_6_smooth_2_4::SetParams (include/rumd/PairPotential.h:232-246):
// c2, c4 from Rcut (in units of sigma) in double, stored as float.
ORC_API void orc_smooth_set_params(int ntypes, float* params, int i, int j,
                                   float sigma, float epsilon, float rcut) {
  float row[NP];
  std::memset(row, 0, sizeof(row));
  row[0] = rcut * sigma;
  row[1] = 1.0f / (sigma * sigma);
  row[2] = 4.0f * epsilon;
  row[3] = (float)(48. * std::pow((double)rcut, -14.0) - 15. * std::pow((double)rcut, -8.));
  row[4] = (float)(6. * std::pow((double)rcut, -10.0) - 21. * std::pow((double)rcut, -16.));
  store_row(ntypes, params, i, j, row, smooth_2_4_f32);
}

// Pot_IPL_n::SetParams (include/rumd/PairPotential.h:616-628).
ORC_API void orc_ipl_n_set_params(int ntypes, float* params, int i, int j, float n,
                                  float sigma, float epsilon, float rcut) {
  float row[NP];
  std::memset(row, 0, sizeof(row));
  row[0] = rcut * sigma;
  row[1] = 1.f / (sigma * sigma);
  row[2] = epsilon;
  row[3] = n;
  store_row(ntypes, params, i, j, row, ipl_n_f32);
}

// ---------------------------------------------------------------------------
// Box arithmetic
// ---------------------------------------------------------------------------

// Min-image component: dr -= L*rint(dr/L).  |rint| <= 1 for wrapped
// coordinates, so L*k is exact and the fused and unfused forms agree.
static inline float mi_f32(float dr, float L, float invL) {
  return std::fmaf(-L, std::rintf(dr * invL), dr);
}

// Squared distance as the device build of calculateDistance evaluates
// dx*dx + dy*dy + dz*dz with multiply-add contraction.
static inline float dist2_ref(float dx, float dy, float dz) {
  return std::fmaf(dz, dz, std::fmaf(dx, dx, dy * dy));
}

static inline int cell_coord_ref(float x, float invL, int nc) {
  float scaled = std::fmaf(x, invL, 0.5f);
  int c = (int)((float)nc * scaled);
  if (c == nc) c -= 1;
  else if (c < 0) c = 0;
  return c;
}

// Squared minimum-image distances of n pairs (calculateDistance).
ORC_API void orc_dist2(int n, const float* a4, const float* b4, const float* L, float* out) {
  float invL[3] = {1.f / L[0], 1.f / L[1], 1.f / L[2]};
  for (int i = 0; i < n; ++i)
    out[i] = dist2_ref(mi_f32(a4[4 * i] - b4[4 * i], L[0], invL[0]),
                       mi_f32(a4[4 * i + 1] - b4[4 * i + 1], L[1], invL[1]),
                       mi_f32(a4[4 * i + 2] - b4[4 * i + 2], L[2], invL[2]));
}

// NeighborList::CalculateNBL_Sorting cell grid: max(floor(2L/(rc+skin)), 5).
ORC_API void orc_cell_grid(const float* L, float max_cut, float skin, int* nc) {
  for (int d = 0; d < 3; ++d) {
    int n = (int)std::floor(2 * L[d] / (max_cut + skin));
    nc[d] = n < 5 ? 5 : n;
  }
}

// calculateCellIndices: linear cell key cx + cy*nx + cz*nx*ny.
ORC_API void orc_cell_keys(int n, const float* pos4, const float* L, const int* nc, int* keys) {
  float invL[3] = {1.f / L[0], 1.f / L[1], 1.f / L[2]};
  for (int i = 0; i < n; ++i) {
    int cx = cell_coord_ref(pos4[4 * i + 0], invL[0], nc[0]);
    int cy = cell_coord_ref(pos4[4 * i + 1], invL[1], nc[1]);
    int cz = cell_coord_ref(pos4[4 * i + 2], invL[2], nc[2]);
    keys[i] = cx + cy * nc[0] + cz * nc[0] * nc[1];
  }
}

// thrust::sort_by_key(keys, iota) is a stable radix sort: sorted slot s holds
// the old index old_index[s], ties kept in ascending old index.
ORC_API void orc_stable_sort_perm(int n, const int* keys, int ncells, unsigned* old_index) {
  std::vector<int> cnt(ncells + 1, 0);
  for (int i = 0; i < n; ++i) cnt[keys[i] + 1]++;
  for (int c = 0; c < ncells; ++c) cnt[c + 1] += cnt[c];
  for (int i = 0; i < n; ++i) old_index[cnt[keys[i]]++] = (unsigned)i;
}

// calculateNBL_CellsSorted on already-sorted positions.  Entries are sorted
// indices in the reference's scan order (dz, dy, dx, then ascending j).
// nbl is row-major [n][max_nbrs]. Returns 1 if any particle overflowed
// (count >= max_nbrs, the reference's "one spare slot" rule).
ORC_API int orc_nbl_build_cells(int n, const float* pos4s, const float* L, const int* nc,
                                int ntypes, const float* params, float skin, int max_nbrs,
                                unsigned* counts, unsigned* nbl) {
  float invL[3] = {1.f / L[0], 1.f / L[1], 1.f / L[2]};
  int ncell = nc[0] * nc[1] * nc[2];
  std::vector<int> keys(n), start(ncell, 0), end(ncell, -1);
  orc_cell_keys(n, pos4s, L, nc, keys.data());
  for (int i = 0; i < n; ++i) {
    if (i == 0 || keys[i - 1] != keys[i]) start[keys[i]] = i;
    if (i == n - 1 || keys[i + 1] != keys[i]) end[keys[i]] = i;
  }
  std::vector<float> cs2(ntypes * ntypes);
  for (int k = 0; k < ntypes * ntypes; ++k) {
    float c = params[k * NP] + skin;
    cs2[k] = c * c;
  }
  int overflow = 0;
  for (int i = 0; i < n; ++i) {
    const float* ri = &pos4s[4 * i];
    int ti; std::memcpy(&ti, &ri[3], 4);
    int cx = cell_coord_ref(ri[0], invL[0], nc[0]);
    int cy = cell_coord_ref(ri[1], invL[1], nc[1]);
    int cz = cell_coord_ref(ri[2], invL[2], nc[2]);
    int count = 0;
    bool full = false;
    for (int dz = -2; dz <= 2 && !full; ++dz) {
      int oz = (cz + dz + nc[2]) % nc[2];
      for (int dy = -2; dy <= 2 && !full; ++dy) {
        int oy = cy + dy;
        if (oy >= nc[1]) oy -= nc[1];
        if (oy < 0) oy += nc[1];
        for (int dx = -2; dx <= 2; ++dx) {
          int ox = cx + dx;
          if (ox < 0) ox += nc[0];
          if (ox >= nc[0]) ox -= nc[0];
          int c = ox + oy * nc[0] + oz * nc[0] * nc[1];
          for (int j = start[c]; j <= end[c]; ++j) {
            if (j == i) continue;
            const float* rj = &pos4s[4 * j];
            int tj; std::memcpy(&tj, &rj[3], 4);
            float ddx = mi_f32(ri[0] - rj[0], L[0], invL[0]);
            float ddy = mi_f32(ri[1] - rj[1], L[1], invL[1]);
            float ddz = mi_f32(ri[2] - rj[2], L[2], invL[2]);
            float d2 = dist2_ref(ddx, ddy, ddz);
            if (d2 < cs2[ti * ntypes + tj]) {
              if (count < max_nbrs) nbl[(size_t)i * max_nbrs + count++] = (unsigned)j;
              else { full = true; break; }
            }
          }
        }
      }
    }
    counts[i] = (unsigned)count;
    if (count >= max_nbrs) overflow = 1;
  }
  return overflow;
}

// All-pairs list (calculateNBL_N2 criterion), ascending j.
ORC_API int orc_nbl_build_n2(int n, const float* pos4, const float* L, int ntypes,
                             const float* params, float skin, int max_nbrs,
                             unsigned* counts, unsigned* nbl) {
  float invL[3] = {1.f / L[0], 1.f / L[1], 1.f / L[2]};
  std::vector<float> cs2(ntypes * ntypes);
  for (int k = 0; k < ntypes * ntypes; ++k) {
    float c = params[k * NP] + skin;
    cs2[k] = c * c;
  }
  int overflow = 0;
#pragma omp parallel for schedule(static) reduction(| : overflow)
  for (int i = 0; i < n; ++i) {
    const float* ri = &pos4[4 * i];
    int ti; std::memcpy(&ti, &ri[3], 4);
    int count = 0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const float* rj = &pos4[4 * j];
      int tj; std::memcpy(&tj, &rj[3], 4);
      float d2 = dist2_ref(mi_f32(ri[0] - rj[0], L[0], invL[0]),
                           mi_f32(ri[1] - rj[1], L[1], invL[1]),
                           mi_f32(ri[2] - rj[2], L[2], invL[2]));
      if (d2 < cs2[ti * ntypes + tj]) {
        if (count < max_nbrs) nbl[(size_t)i * max_nbrs + count] = (unsigned)j;
        count++;
      }
    }
    counts[i] = (unsigned)(count < max_nbrs ? count : max_nbrs);
    if (count >= max_nbrs) overflow = 1;
  }
  return overflow;
}

// NeighborList::UpdateNBlist capacity rule (src/NeighborList.cu:595-606).
ORC_API unsigned orc_max_nbrs_estimate(unsigned n, float max_cut, float skin, double volume) {
  if (n < 10000) return n;
  float rm_sk = max_cut + skin;
  unsigned est = (unsigned)(1.5 * (4. / 3.) * M_PI * rm_sk * rm_sk * rm_sk * n / volume);
  if (est < 50) est = 50;
  return est;
}

// ---------------------------------------------------------------------------
// Pair forces
// ---------------------------------------------------------------------------

enum { ORC_POT_LJ_12_6 = 0, ORC_POT_LJ_12_6_SMOOTH_2_4 = 1, ORC_POT_IPL_N = 2 };

// The pair functions in double at squared distance d2 for a parameter row of
// the reference layout: F = s d, energy u.
//   LJ 12-6          Pot_IPL_12_6::ComputeInteraction  PairPotential.h:161-168
//   LJ 12-6 smooth   Pot_LJ_12_6_smooth_2_4             PairPotential.h:248-255
//   IPL n            Pot_IPL_n                          PairPotential.h:630-636
static void pair_f64(int kind, double d2, const float* p, double* s, double* u) {
  if (kind == ORC_POT_LJ_12_6) {
    double i2 = 1. / d2, i6 = i2 * i2 * i2, a12 = p[1], a6 = p[2];
    *s = i6 * i2 * (12. * a12 * i6 + 6. * a6);
    *u = i6 * (a12 * i6 + a6);
  } else if (kind == ORC_POT_LJ_12_6_SMOOTH_2_4) {
    double is2 = p[1], a = p[2], c2 = p[3], c4 = p[4];
    double D2 = d2 * is2, i2 = 1. / D2, i6 = i2 * i2 * i2;
    *s = a * is2 * (i2 * i6 * (12. * i6 - 6.) - 2. * c2 - 4. * c4 * D2);
    *u = a * (i6 * (i6 - 1.) + c2 * D2 + c4 * D2 * D2);
  } else {
    double is2 = p[1], eps = p[2], nn = p[3];
    double i2 = 1. / (d2 * is2), tn = std::pow(i2, 0.5 * nn);
    *s = is2 * eps * nn * tn * i2;
    *u = eps * tn;
  }
}

// FP64 pair sum over all j within Rcut (minimum image), every pair visited
// from both sides as the reference's full list does.  u is halved per
// particle (Calcf: f.w *= 0.5), w = sum d^2 s (w.w), forces F_i = sum s*d.
// Uses a cell list with cells >= max cutoff, or all pairs for small boxes.
// The cut-off terms (fij, PairPotential.h:1208-1221) use s(rc), u(rc) of the
// same pair function in double.
// The same sum with the per-particle stress of fij's STR branch
// (PairPotential.h:1232-1241): sts6[6 i + (xx, yy, zz, yz, xz, xy)] =
// -sum_j d_a d_b s over the pairs within the cut-off (RUMD keeps xx, yy, zz,
// yz in sts and xz, xy in w.y, w.z).  sts6 may be null.
// fp32_cut: a pair is in the sum when the reference's FP32 arithmetic puts
// it inside the cut-off (dist.w < param[0]*param[0] in float, fij,
// PairPotential.h:1206-1207) rather than when the FP64 distance does.  With
// the NS and SP cut-offs the pair force does not vanish at rc, so a pair
// within a rounding error of rc changes the sum; this option makes the FP64
// oracle sum exactly the pairs the reference sums.
ORC_API void orc_forces_stress_f64_pot(int n, const double* pos3, const int* type, const double* L,
                                       int ntypes, const float* params, int cutoff, int potential,
                                       double* f3, double* u, double* w, double* sts6, int fp32_cut);

ORC_API void orc_forces_f64_pot(int n, const double* pos3, const int* type, const double* L,
                                int ntypes, const float* params, int cutoff, int potential,
                                double* f3, double* u, double* w) {
  orc_forces_stress_f64_pot(n, pos3, type, L, ntypes, params, cutoff, potential, f3, u, w, nullptr, 0);
}

ORC_API void orc_forces_stress_f64_pot(int n, const double* pos3, const int* type, const double* L,
                                       int ntypes, const float* params, int cutoff, int potential,
                                       double* f3, double* u, double* w, double* sts6, int fp32_cut) {
  const float Lf[3] = {(float)L[0], (float)L[1], (float)L[2]};
  const float iLf[3] = {1.f / Lf[0], 1.f / Lf[1], 1.f / Lf[2]};
  double invL[3] = {1. / L[0], 1. / L[1], 1. / L[2]};
  double maxc = 0;
  for (int k = 0; k < ntypes * ntypes; ++k) maxc = std::max(maxc, (double)params[k * NP]);
  int nc[3];
  bool use_cells = true;
  for (int d = 0; d < 3; ++d) {
    nc[d] = (int)std::floor(L[d] / maxc);
    if (nc[d] < 3) use_cells = false;
  }
  std::vector<int> head, next;
  std::vector<int> cell_of(n);
  if (use_cells) {
    head.assign(nc[0] * nc[1] * nc[2], -1);
    next.assign(n, -1);
    for (int i = 0; i < n; ++i) {
      int c[3];
      for (int d = 0; d < 3; ++d) {
        double s = pos3[3 * i + d] * invL[d] + 0.5;
        s -= std::floor(s);
        c[d] = (int)(s * nc[d]);
        if (c[d] >= nc[d]) c[d] = nc[d] - 1;
      }
      int ci = c[0] + nc[0] * (c[1] + nc[1] * c[2]);
      cell_of[i] = ci;
      next[i] = head[ci];
      head[ci] = i;
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    double fx = 0, fy = 0, fz = 0, ui = 0, wi = 0;
    double sxx = 0, syy = 0, szz = 0, syz = 0, sxz = 0, sxy = 0;
    auto pair = [&](int j) {
      if (j == i) return;
      double dx = pos3[3 * i] - pos3[3 * j];
      double dy = pos3[3 * i + 1] - pos3[3 * j + 1];
      double dz = pos3[3 * i + 2] - pos3[3 * j + 2];
      dx -= L[0] * std::nearbyint(dx * invL[0]);
      dy -= L[1] * std::nearbyint(dy * invL[1]);
      dz -= L[2] * std::nearbyint(dz * invL[2]);
      double d2 = dx * dx + dy * dy + dz * dz;
      const float* p = &params[(type[i] * ntypes + type[j]) * NP];
      double rc = p[0];
      bool in = d2 < rc * rc;
      if (fp32_cut) {
        const float fx = mi_f32((float)pos3[3 * i] - (float)pos3[3 * j], Lf[0], iLf[0]);
        const float fy = mi_f32((float)pos3[3 * i + 1] - (float)pos3[3 * j + 1], Lf[1], iLf[1]);
        const float fz = mi_f32((float)pos3[3 * i + 2] - (float)pos3[3 * j + 2], Lf[2], iLf[2]);
        in = dist2_ref(fx, fy, fz) < p[0] * p[0];
      }
      if (in) {
        double s, uu;
        pair_f64(potential, d2, p, &s, &uu);
        if (cutoff != ORC_NS) {
          double sc, uc;
          pair_f64(potential, rc * rc, p, &sc, &uc);
          if (cutoff == ORC_SP) {
            uu -= uc;
          } else {
            double r = std::sqrt(d2);
            s -= sc * rc / r;
            uu += sc * rc * (r - rc) - uc;
          }
        }
        fx += dx * s; fy += dy * s; fz += dz * s;
        ui += uu; wi += d2 * s;
        sxx -= dx * dx * s; syy -= dy * dy * s; szz -= dz * dz * s;
        syz -= dy * dz * s; sxz -= dx * dz * s; sxy -= dx * dy * s;
      }
    };
    if (use_cells) {
      int ci = cell_of[i];
      int cx = ci % nc[0], cy = (ci / nc[0]) % nc[1], cz = ci / (nc[0] * nc[1]);
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int ox = (cx + dx + nc[0]) % nc[0], oy = (cy + dy + nc[1]) % nc[1], oz = (cz + dz + nc[2]) % nc[2];
            for (int j = head[ox + nc[0] * (oy + nc[1] * oz)]; j >= 0; j = next[j]) pair(j);
          }
    } else {
      for (int j = 0; j < n; ++j) pair(j);
    }
    f3[3 * i] = fx; f3[3 * i + 1] = fy; f3[3 * i + 2] = fz;
    u[i] = 0.5 * ui; w[i] = wi;
    if (sts6) {
      double* o = sts6 + 6 * (size_t)i;
      o[0] = sxx; o[1] = syy; o[2] = szz; o[3] = syz; o[4] = sxz; o[5] = sxy;
    }
  }
}

ORC_API void orc_forces_f64(int n, const double* pos3, const int* type, const double* L,
                            int ntypes, const float* params, int cutoff,
                            double* f3, double* u, double* w) {
  orc_forces_f64_pot(n, pos3, type, L, ntypes, params, cutoff, ORC_POT_LJ_12_6, f3, u, w);
}

// FP32 reference-arithmetic force sum over a row-major list (fij + Calcf with
// tp = 1: neighbours accumulated in list order, then f.w *= 0.5).
ORC_API void orc_forces_f32(int n, const float* pos4, const float* L, int ntypes,
                            const float* params, int cutoff, const unsigned* counts,
                            const unsigned* nbl, int max_nbrs, float* f4, float* w) {
  float invL[3] = {1.f / L[0], 1.f / L[1], 1.f / L[2]};
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const float* ri = &pos4[4 * i];
    int ti; std::memcpy(&ti, &ri[3], 4);
    float fx = 0, fy = 0, fz = 0, fw = 0, ww = 0;
    for (unsigned k = 0; k < counts[i]; ++k) {
      unsigned j = nbl[(size_t)i * max_nbrs + k];
      const float* rj = &pos4[4 * j];
      int tj; std::memcpy(&tj, &rj[3], 4);
      const float* p = &params[(ti * ntypes + tj) * NP];
      float dx = mi_f32(ri[0] - rj[0], L[0], invL[0]);
      float dy = mi_f32(ri[1] - rj[1], L[1], invL[1]);
      float dz = mi_f32(ri[2] - rj[2], L[2], invL[2]);
      float d2 = dist2_ref(dx, dy, dz);
      if (d2 < p[0] * p[0]) {
        float s = ipl_12_6_f32(d2, p, &fw);
        if (cutoff == ORC_SP) {
          fw -= p[NP - 1];
        } else if (cutoff == ORC_SF) {
          float r = std::sqrt(d2);
          s -= p[NP - 2] / r;
          fw += p[NP - 2] * (r - p[0]) - p[NP - 1];
        }
        fx += dx * s; fy += dy * s; fz += dz * s;
        ww += d2 * s;
      }
    }
    f4[4 * i] = fx; f4[4 * i + 1] = fy; f4[4 * i + 2] = fz; f4[4 * i + 3] = fw * 0.5f;
    w[i] = ww;
  }
}

// ---------------------------------------------------------------------------
// Full MD loop (CPU baseline and trajectory oracle)
// ---------------------------------------------------------------------------
//
// One step, as Simulation.Run does it (Python/rumd/Simulation.py:579-598):
//   momentum reset when step % reset_interval == 0,
//   CalcF: rebuild list if any particle moved more than skin/2 since the last
//          build (sort by cell key, sorted cell scan), then forces,
//   Integrate: Nose-Hoover leap-frog, wrap, images, thermostat update.
// R = float gives the reference's FP32 arithmetic, R = double the FP64 oracle.
// Per-step outputs (optional): pe(t), W(t), KE(t) (leap-frog), xi after step.

template <class R> struct MDState {
  int n, ntypes, cutoff;
  R L[3], invL[3];
  float Lf[3];
  std::vector<R> r, v, f;      // 3 per particle (v.w = 1/m kept in invm)
  std::vector<R> invm;
  std::vector<int> type, im;   // images, 3 per particle
  std::vector<unsigned> uidx;  // original index of sorted slot
  std::vector<R> last_r;
  std::vector<R> u, w;
  std::vector<unsigned> counts, nbl;
  int max_nbrs, nc[3];
  const float* params;
  float skin;
  // FP64 mode only: s(rc) rc and u(rc) per type pair, computed in double from
  // rc, A12, A6 (what CopyParamsToGPU computes in a changeToDouble.sh build)
  std::vector<double> cs64, cu64;
};

template <class R> static inline R mi(R dr, R L, R invL) {
  if (sizeof(R) == 4) return (R)mi_f32((float)dr, (float)L, (float)invL);
  return dr - L * std::nearbyint(dr * invL);
}
template <class R> static inline R d2of(R dx, R dy, R dz) {
  if (sizeof(R) == 4) return (R)dist2_ref((float)dx, (float)dy, (float)dz);
  return dx * dx + dy * dy + dz * dz;
}

template <class R> static int md_rebuild(MDState<R>& S) {
  int n = S.n;
  // keys on float positions (the reference sorts FP32 positions)
  std::vector<float> p4(4 * n);
  for (int i = 0; i < n; ++i) {
    p4[4 * i] = (float)S.r[3 * i]; p4[4 * i + 1] = (float)S.r[3 * i + 1]; p4[4 * i + 2] = (float)S.r[3 * i + 2];
    std::memcpy(&p4[4 * i + 3], &S.type[i], 4);
  }
  int ncell = S.nc[0] * S.nc[1] * S.nc[2];
  std::vector<int> keys(n);
  orc_cell_keys(n, p4.data(), S.Lf, S.nc, keys.data());
  std::vector<unsigned> old(n);
  orc_stable_sort_perm(n, keys.data(), ncell, old.data());
  // permute r, v, invm, type, im, uidx
  auto perm3 = [&](std::vector<R>& a) {
    std::vector<R> t(a.size());
    for (int s = 0; s < n; ++s) for (int d = 0; d < 3; ++d) t[3 * s + d] = a[3 * old[s] + d];
    a.swap(t);
  };
  perm3(S.r); perm3(S.v);
  {
    std::vector<R> t(n); for (int s = 0; s < n; ++s) t[s] = S.invm[old[s]]; S.invm.swap(t);
    std::vector<int> ty(n); for (int s = 0; s < n; ++s) ty[s] = S.type[old[s]]; S.type.swap(ty);
    std::vector<int> ti(3 * n);
    for (int s = 0; s < n; ++s) for (int d = 0; d < 3; ++d) ti[3 * s + d] = S.im[3 * old[s] + d];
    S.im.swap(ti);
    std::vector<unsigned> tu(n); for (int s = 0; s < n; ++s) tu[s] = S.uidx[old[s]]; S.uidx.swap(tu);
  }
  int ntypes = S.ntypes;
  std::vector<int> start(ncell, 0), end(ncell, -1);
  for (int s = 0; s < n; ++s) {
    int k = keys[old[s]];
    if (s == 0 || keys[old[s - 1]] != k) start[k] = s;
    if (s == n - 1 || keys[old[s + 1]] != k) end[k] = s;
  }
  std::vector<R> cs2(ntypes * ntypes);
  for (int k = 0; k < ntypes * ntypes; ++k) {
    if (sizeof(R) == 4) { float c = S.params[k * NP] + S.skin; cs2[k] = c * c; }
    else { double c = (double)S.params[k * NP] + (double)S.skin; cs2[k] = c * c; }
  }
  int overflow = 0;
  const int* nc = S.nc;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : overflow)
  for (int i = 0; i < n; ++i) {
    int cx = cell_coord_ref((float)S.r[3 * i], 1.f / S.Lf[0], nc[0]);
    int cy = cell_coord_ref((float)S.r[3 * i + 1], 1.f / S.Lf[1], nc[1]);
    int cz = cell_coord_ref((float)S.r[3 * i + 2], 1.f / S.Lf[2], nc[2]);
    int ti = S.type[i];
    unsigned count = 0;
    for (int dz = -2; dz <= 2; ++dz) {
      int oz = (cz + dz + nc[2]) % nc[2];
      for (int dy = -2; dy <= 2; ++dy) {
        int oy = (cy + dy + nc[1]) % nc[1];
        for (int dx = -2; dx <= 2; ++dx) {
          int ox = (cx + dx + nc[0]) % nc[0];
          int c = ox + oy * nc[0] + oz * nc[0] * nc[1];
          for (int j = start[c]; j <= end[c]; ++j) {
            if (j == i) continue;
            R ddx = mi<R>(S.r[3 * i] - S.r[3 * j], S.L[0], S.invL[0]);
            R ddy = mi<R>(S.r[3 * i + 1] - S.r[3 * j + 1], S.L[1], S.invL[1]);
            R ddz = mi<R>(S.r[3 * i + 2] - S.r[3 * j + 2], S.L[2], S.invL[2]);
            if (d2of<R>(ddx, ddy, ddz) < cs2[ti * ntypes + S.type[j]]) {
              if ((int)count < S.max_nbrs) S.nbl[(size_t)i * S.max_nbrs + count] = (unsigned)j;
              count++;
            }
          }
        }
      }
    }
    if ((int)count >= S.max_nbrs) overflow = 1;
    S.counts[i] = (unsigned)std::min<unsigned>(count, S.max_nbrs);
    for (int d = 0; d < 3; ++d) S.last_r[3 * i + d] = S.r[3 * i + d];
  }
  return overflow;
}

template <class R> static void md_forces(MDState<R>& S) {
  int n = S.n, ntypes = S.ntypes;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    R fx = 0, fy = 0, fz = 0, fw = 0, ww = 0;
    int ti = S.type[i];
    for (unsigned k = 0; k < S.counts[i]; ++k) {
      unsigned j = S.nbl[(size_t)i * S.max_nbrs + k];
      const float* p = &S.params[(ti * ntypes + S.type[j]) * NP];
      R dx = mi<R>(S.r[3 * i] - S.r[3 * j], S.L[0], S.invL[0]);
      R dy = mi<R>(S.r[3 * i + 1] - S.r[3 * j + 1], S.L[1], S.invL[1]);
      R dz = mi<R>(S.r[3 * i + 2] - S.r[3 * j + 2], S.L[2], S.invL[2]);
      R d2 = d2of<R>(dx, dy, dz);
      R rc = p[0];
      if (d2 < rc * rc) {
        R s;
        if (sizeof(R) == 4) {
          float fwf = (float)fw;
          s = ipl_12_6_f32((float)d2, p, &fwf);
          fw = fwf;
        } else {
          R i2 = R(1) / d2, i6 = i2 * i2 * i2, t = (R)p[1] * i6;
          s = i6 * i2 * (R(12) * t + R(6) * (R)p[2]);
          fw += i6 * (t + (R)p[2]);
        }
        const int pk = ti * ntypes + S.type[j];
        const R cs = sizeof(R) == 8 ? (R)S.cs64[pk] : (R)p[NP - 2];
        const R cu = sizeof(R) == 8 ? (R)S.cu64[pk] : (R)p[NP - 1];
        if (S.cutoff == ORC_SP) {
          fw -= cu;
        } else if (S.cutoff == ORC_SF) {
          R r = std::sqrt(d2);
          s -= cs / r;
          fw += cs * (r - rc) - cu;
        }
        fx += dx * s; fy += dy * s; fz += dz * s;
        ww += d2 * s;
      }
    }
    S.f[3 * i] = fx; S.f[3 * i + 1] = fy; S.f[3 * i + 2] = fz;
    S.u[i] = fw * R(0.5);
    S.w[i] = ww;
  }
}

// Runs nsteps of Simulation.Run.  Arrays are in ORIGINAL particle order on
// entry and on exit (pos4: x,y,z,type-bits; vel4: vx,vy,vz,1/m; im3 int).
// Per-step outputs: energies[4*k + {0,1,2,3}] = pe(t), W(t) = sum w/6,
// KE(t) (leap-frog average), xi after the step.  Returns the number of list
// rebuilds, or -1 on list overflow.
template <class R>
static int md_run(int n, float* pos4, float* vel4, int* im3, const float* L, int ntypes,
                  const float* params, int cutoff, float skin, float dt, double T,
                  double tau, double* xi_io, int thermostat_on, int nsteps,
                  int reset_interval, int max_nbrs, double* energies, double* f_out) {
  MDState<R> S;
  S.n = n; S.ntypes = ntypes; S.cutoff = cutoff; S.params = params; S.skin = skin;
  for (int d = 0; d < 3; ++d) {
    S.Lf[d] = L[d];
    S.L[d] = (R)L[d];
    S.invL[d] = (sizeof(R) == 4) ? (R)(1.f / L[d]) : R(1) / (R)L[d];
  }
  S.r.resize(3 * n); S.v.resize(3 * n); S.f.assign(3 * n, 0); S.invm.resize(n);
  S.type.resize(n); S.im.resize(3 * n); S.uidx.resize(n); S.last_r.resize(3 * n);
  S.u.assign(n, 0); S.w.assign(n, 0);
  float maxc = 0;
  for (int k = 0; k < ntypes * ntypes; ++k) maxc = std::max(maxc, params[k * NP]);
  orc_cell_grid(L, maxc, skin, S.nc);
  S.max_nbrs = max_nbrs;
  S.counts.assign(n, 0); S.nbl.assign((size_t)n * max_nbrs, 0);
  for (int i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) { S.r[3 * i + d] = pos4[4 * i + d]; S.v[3 * i + d] = vel4[4 * i + d]; S.im[3 * i + d] = im3[3 * i + d]; }
    S.invm[i] = vel4[4 * i + 3];
    std::memcpy(&S.type[i], &pos4[4 * i + 3], 4);
    S.uidx[i] = (unsigned)i;
  }
  S.cs64.resize(ntypes * ntypes);
  S.cu64.resize(ntypes * ntypes);
  for (int k = 0; k < ntypes * ntypes; ++k) {
    const double rc = params[k * NP], a12 = params[k * NP + 1], a6 = params[k * NP + 2];
    const double i2 = 1.0 / (rc * rc), i6 = i2 * i2 * i2;
    S.cu64[k] = i6 * (a12 * i6 + a6);
    S.cs64[k] = i6 * i2 * (12.0 * a12 * i6 + 6.0 * a6) * rc;
  }
  double xi = *xi_io;
  // omega^2 = 4 pi^2 / tau^2: a float in the reference, a double in its FP64 build
  const double omega2 = sizeof(R) == 4 ? (double)(float)(4. * M_PI * M_PI / (tau * tau))
                                       : 4. * M_PI * M_PI / (tau * tau);
  const int dof = 3 * n - 3;
  const float s2_4 = (float)(0.25 * skin * skin);
  int rebuilds = 0;
  bool need = true;
  for (int step = 0; step < nsteps; ++step) {
    if (reset_interval > 0 && step % reset_interval == 0) {
      double P[3] = {0, 0, 0}, M = 0;
      for (int i = 0; i < n; ++i) {
        double m = 1.0 / (double)S.invm[i];
        for (int d = 0; d < 3; ++d) P[d] += m * (double)S.v[3 * i + d];
        M += m;
      }
      for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) S.v[3 * i + d] -= (R)(P[d] / M);
    }
    if (!need) {
      for (int i = 0; i < n && !need; ++i) {
        R dx = mi<R>(S.r[3 * i] - S.last_r[3 * i], S.L[0], S.invL[0]);
        R dy = mi<R>(S.r[3 * i + 1] - S.last_r[3 * i + 1], S.L[1], S.invL[1]);
        R dz = mi<R>(S.r[3 * i + 2] - S.last_r[3 * i + 2], S.L[2], S.invL[2]);
        if (d2of<R>(dx, dy, dz) > (R)s2_4) need = true;
      }
    }
    if (need) {
      if (md_rebuild(S)) return -1;
      rebuilds++;
      need = false;
    }
    md_forces(S);
    double pe = 0, W = 0, ke_t = 0, ke2 = 0;
    R factor = thermostat_on ? (R)(0.5 * xi * (double)dt) : R(0);
    R plus = R(1) / (R(1) + factor), minus = R(1) - factor;
    if (sizeof(R) == 4) {
      // as the device build contracts it: factor = (xi/2) dt is fused into
      // both sums, plus = 1 / fma(xi/2, dt, 1), minus = fma(-xi/2, dt, 1)
      const float h = thermostat_on ? 0.5f * (float)xi : 0.f;
      plus = (R)(1.f / std::fmaf(h, dt, 1.f));
      minus = (R)std::fmaf(-h, dt, 1.f);
    }
#pragma omp parallel for schedule(static) reduction(+ : pe, W, ke_t, ke2)
    for (int i = 0; i < n; ++i) {
      pe += (double)S.u[i];
      W += (double)S.w[i];
      double vb = 0, vf = 0;
      R im_ = S.invm[i];
      for (int d = 0; d < 3; ++d) {
        R vo = S.v[3 * i + d];
        R vn, x, k;
        if (sizeof(R) == 4) {
          // integrateNVTAlgorithm as the device build contracts it:
          // v = plus * fma((1/m) f, dt, minus v);  r = fma(v, dt, r)
          const float mf = (float)im_ * (float)S.f[3 * i + d];
          vn = (R)((float)plus * std::fmaf(mf, dt, (float)minus * (float)vo));
          x = (R)std::fmaf((float)vn, dt, (float)S.r[3 * i + d]);
          k = (R)std::rintf((float)x * (float)S.invL[d]);
          x = (R)std::fmaf(-(float)S.L[d], (float)k, (float)x);
        } else {
          vn = plus * (minus * vo + im_ * S.f[3 * i + d] * (R)dt);
          x = S.r[3 * i + d] + vn * (R)dt;
          k = std::nearbyint(x * S.invL[d]);
          x = x - S.L[d] * k;
        }
        S.v[3 * i + d] = vn;
        vb += (double)vo * (double)vo;
        vf += (double)vn * (double)vn;
        S.r[3 * i + d] = x;
        S.im[3 * i + d] += (int)k;
      }
      double m = 1.0 / (double)im_;
      ke_t += 0.25 * m * (vb + vf);
      ke2 += m * vf;
    }
    if (thermostat_on) {
      double dev = ke2 / ((double)dof * T) - 1.0;
      if (dev > 10.0) dev = 10.0;
      xi += (double)dt * (double)omega2 * dev;
    }
    if (energies) {
      energies[4 * step + 0] = pe;
      energies[4 * step + 1] = W / 6.0;
      energies[4 * step + 2] = ke_t;
      energies[4 * step + 3] = xi;
    }
    for (int i = 0; i < n && !need; ++i) {
      R dx = mi<R>(S.r[3 * i] - S.last_r[3 * i], S.L[0], S.invL[0]);
      R dy = mi<R>(S.r[3 * i + 1] - S.last_r[3 * i + 1], S.L[1], S.invL[1]);
      R dz = mi<R>(S.r[3 * i + 2] - S.last_r[3 * i + 2], S.L[2], S.invL[2]);
      if (d2of<R>(dx, dy, dz) > (R)s2_4) need = true;
    }
  }
  *xi_io = xi;
  for (int s = 0; s < n; ++s) {
    unsigned o = S.uidx[s];
    for (int d = 0; d < 3; ++d) {
      pos4[4 * o + d] = (float)S.r[3 * s + d];
      vel4[4 * o + d] = (float)S.v[3 * s + d];
      im3[3 * o + d] = S.im[3 * s + d];
      if (f_out) f_out[3 * o + d] = (double)S.f[3 * s + d];
    }
  }
  return rebuilds;
}

ORC_API int orc_md_run_f32(int n, float* pos4, float* vel4, int* im3, const float* L, int ntypes,
                           const float* params, int cutoff, float skin, float dt, double T,
                           double tau, double* xi_io, int thermostat_on, int nsteps,
                           int reset_interval, int max_nbrs, double* energies, double* f_out) {
  return md_run<float>(n, pos4, vel4, im3, L, ntypes, params, cutoff, skin, dt, T, tau, xi_io,
                       thermostat_on, nsteps, reset_interval, max_nbrs, energies, f_out);
}

ORC_API int orc_md_run_f64(int n, float* pos4, float* vel4, int* im3, const float* L, int ntypes,
                           const float* params, int cutoff, float skin, float dt, double T,
                           double tau, double* xi_io, int thermostat_on, int nsteps,
                           int reset_interval, int max_nbrs, double* energies, double* f_out) {
  return md_run<double>(n, pos4, vel4, im3, L, ntypes, params, cutoff, skin, dt, T, tau, xi_io,
                        thermostat_on, nsteps, reset_interval, max_nbrs, energies, f_out);
}

ORC_API int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

ORC_API void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
