/*
 * Precision-templated body of the CPU oracle (test infrastructure only).
 * Included twice by dem_oracle.c with REAL/SFX/ONE... defined.
 * Loops over particles are OpenMP-parallel: each iteration writes only its
 * own particle's slots and force, exactly as one CUDA thread of the
 * reference does, so results do not depend on the thread count.
 */

#define NORM3(x, y, z) NORM3_RN(x, y, z)
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* float -> unsigned conversion with the saturation of the GPU's cvt.rzi.u32 */
static inline uint32_t FN(to_u32)(REAL v) {
  if (!(v > 0)) return 0u;
  if (v >= (REAL)4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

void FN(orc_cell_distribution)(const REAL* R, uint32_t N, REAL inv_a, uint32_t nx, uint32_t ny,
                               uint32_t nz, uint32_t* CI, uint32_t* CIs, uint32_t* pnC) {
  /* md_calculate_cell.cu:22-36 */
  for (uint32_t idx = 0; idx < N; ++idx) {
    uint32_t ix = FN(to_u32)(FLOOR(R[idx] * inv_a));
    uint32_t iy = FN(to_u32)(FLOOR(R[idx + N] * inv_a));
    uint32_t iz = FN(to_u32)(FLOOR(R[idx + 2 * N] * inv_a));
    CI[idx] = ix + iy * nx + iz * ny * nx;
  }
  /* cub::DeviceRadixSort::SortPairs (md_cell_distribution.cu:146-165): a stable
   * ascending sort of (cell, particle) pairs, restated as a counting sort. */
  uint64_t CN = (uint64_t)nx * ny * nz;
  uint32_t* cnt = (uint32_t*)calloc(CN + 1, sizeof(uint32_t));
  for (uint32_t i = 0; i < N; ++i) cnt[CI[i] < CN ? CI[i] + 1 : CN]++;
  for (uint64_t c = 0; c < CN; ++c) cnt[c + 1] += cnt[c];
  /* cells outside the grid cannot occur for valid samples; they sort last */
  uint32_t* pos = (uint32_t*)malloc((CN + 1) * sizeof(uint32_t));
  memcpy(pos, cnt, (CN + 1) * sizeof(uint32_t));
  uint32_t* keys = CIs;
  uint32_t* vals = CIs + N;
  uint32_t tail = cnt[CN];
  for (uint32_t i = 0; i < N; ++i) {
    uint32_t c = CI[i];
    uint32_t p = (c < CN) ? pos[c]++ : tail++;
    keys[p] = c;
    vals[p] = i;
  }
  /* md_cell_distribution.cu:171 memset + md_calculate_cell.cu:43-75.  The
   * reference's run-length scan may step into the value half past the last key;
   * the oracle records the true run length. */
  memset(pnC, 0, 2 * CN * sizeof(uint32_t));
  for (uint32_t idx = 0; idx < N; ++idx) {
    uint32_t c = keys[idx];
    if (c >= CN) continue;
    if (idx == 0 || keys[idx - 1] != c) {
      uint32_t n = 1;
      while (idx + n < N && keys[idx + n] == c) ++n;
      pnC[c] = idx;
      pnC[c + CN] = n;
    }
  }
  free(cnt);
  free(pos);
}

/* The eight-cell "octant" search shared by construct / reconstruct
 * (md_interaction_list_construct.cu:264-304, reconstructbpm.cu:96-134). */
static inline void FN(octant_cells)(const REAL* R, uint32_t N, uint32_t idx, REAL a, REAL inv_a,
                                    uint32_t nx, uint32_t ny, uint32_t cells[8]) {
  uint32_t ix = FN(to_u32)(FLOOR(R[idx] * inv_a));
  uint32_t iy = FN(to_u32)(FLOOR(R[idx + N] * inv_a));
  uint32_t iz = FN(to_u32)(FLOOR(R[idx + 2 * N] * inv_a));
  uint32_t ii = ix + iy * nx + iz * ny * nx;
  int sx = (int)COPYSIGN((REAL)1, R[idx] - ((REAL)ix + (REAL)0.5) * a);
  int sy = (int)COPYSIGN((REAL)1, R[idx + N] - ((REAL)iy + (REAL)0.5) * a);
  int sz = (int)COPYSIGN((REAL)1, R[idx + 2 * N] - ((REAL)iz + (REAL)0.5) * a);
  uint32_t dx = (uint32_t)sx, dy = (uint32_t)sy * nx, dz = (uint32_t)sz * ny * nx;
  cells[0] = ii;
  cells[1] = ii + dx;
  cells[2] = ii + dy;
  cells[3] = ii + dz;
  cells[4] = ii + dx + dy;
  cells[5] = ii + dx + dz;
  cells[6] = ii + dy + dz;
  cells[7] = ii + dx + dy + dz;
}

static inline REAL FN(dist2)(const REAL* R, uint32_t N, uint32_t i, uint32_t j) {
  REAL dx = R[j] - R[i], dy = R[j + N] - R[i + N], dz = R[j + 2 * N] - R[i + 2 * N];
  return (dx * dx + dy * dy) + dz * dz;
}

int64_t FN(orc_il_construct)(const REAL* R, uint32_t N, const uint32_t* CIs, const uint32_t* pnC,
                             uint32_t* IL, uint32_t IonP, REAL a, REAL inv_a, REAL aacut, uint32_t nx,
                             uint32_t ny, uint32_t nz) {
  uint64_t CN = (uint64_t)nx * ny * nz;
  int64_t overflow = 0;
#pragma omp parallel for schedule(static) reduction(+ : overflow)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii, cells[8], nk = 0;
    FN(octant_cells)(R, N, idx, a, inv_a, nx, ny, cells);
    for (int c = 0; c < 8; ++c) {
      uint32_t cc = cells[c];
      if (cc >= CN) continue;
      uint32_t start = pnC[cc], n = pnC[cc + CN];
      for (uint32_t i = 0; i < n; ++i) {
        uint32_t jdx = CIs[start + i + N];
        REAL rr = FN(dist2)(R, N, idx, jdx);
        if (rr < aacut && jdx != idx) {
          if (nk < IonP)
            IL[(uint64_t)idx * IonP + nk] = jdx;
          else
            ++overflow;
          ++nk;
        }
      }
    }
  }
  return overflow;
}

int64_t FN(orc_il_reconstruct_bpm)(const REAL* R, uint32_t N, const uint32_t* CIs, const uint32_t* pnC,
                                   uint32_t* IL, uint32_t* ILtype, uint32_t IonP, REAL a, REAL inv_a,
                                   REAL aacut, uint32_t nx, uint32_t ny, uint32_t nz) {
  uint64_t CN = (uint64_t)nx * ny * nz;
  int64_t overflow = 0;
#pragma omp parallel for schedule(static) reduction(+ : overflow)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii, cells[8];
    FN(octant_cells)(R, N, idx, a, inv_a, nx, ny, cells);
    uint64_t base = (uint64_t)idx * IonP;
    for (int c = 0; c < 8; ++c) {
      uint32_t cc = cells[c];
      if (cc >= CN) continue;
      uint32_t start = pnC[cc], n = pnC[cc + CN];
      /* addnewlinkbpm, md_interaction_list_reconstructbpm.cu:13-46 */
      for (uint32_t i = 0; i < n; ++i) {
        uint32_t jdx = CIs[start + i + N];
        REAL rr = FN(dist2)(R, N, idx, jdx);
        if (rr < aacut && rr > 1e-10) {
          uint64_t kdxfree = 0;
          uint32_t j;
          for (j = 0; j < IonP; ++j) {
            uint32_t kj = IL[base + j];
            if (kdxfree == 0 && kj == ORC_EMPTY) kdxfree = base + j;
            if (kj == jdx) break;
          }
          if (j == IonP) {
            /* kdxfree==0 is also the reference's "no free slot" sentinel: the
             * reference then writes slot 0 of particle 0.  Only the legitimate
             * case (particle 0, slot 0 free) is written here. */
            if (kdxfree == 0 && !(idx == 0 && IL[0] == ORC_EMPTY)) {
              ++overflow;
            } else {
              IL[kdxfree] = jdx;
              ILtype[kdxfree] = 0;
            }
          }
        }
      }
    }
  }
  return overflow;
}

void FN(orc_delete_far_links)(const REAL* R, uint32_t N, uint32_t* IL, uint32_t* ILtype, REAL* Rij,
                              REAL* Oijt, REAL* Mijn, REAL* Mijt, uint32_t IonP, REAL aacut) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    for (uint32_t k = 0; k < IonP; ++k) {
      uint64_t kdx = (uint64_t)idx * IonP + k;
      uint32_t jdx = IL[kdx];
      if (jdx == ORC_EMPTY) continue;
      REAL rr = FN(dist2)(R, N, idx, jdx);
      if (rr > aacut || rr < 1e-10) {
        IL[kdx] = ORC_EMPTY;
        ILtype[kdx] = 0;
        for (int d = 0; d < 3; ++d) {
          Rij[3 * kdx + d] = 0;
          Oijt[3 * kdx + d] = 0;
          Mijn[3 * kdx + d] = 0;
          Mijt[3 * kdx + d] = 0;
        }
      }
    }
  }
}

void FN(orc_construct_bonds)(const REAL* R, uint32_t N, const uint32_t* IL, uint32_t* ILtype,
                             REAL* inv_L0, REAL* Rij, REAL* Oijt, REAL* Mijn, REAL* Mijt,
                             uint32_t IonP, REAL aa_create, const REAL* rad, double gap) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    for (uint32_t k = 0; k < IonP; ++k) {
      uint64_t kdx = (uint64_t)idx * IonP + k;
      uint32_t jdx = IL[kdx];
      if (jdx == ORC_EMPTY) continue;
      REAL rx = R[jdx] - R[idx], ry = R[jdx + N] - R[idx + N], rz = R[jdx + 2 * N] - R[idx + 2 * N];
      REAL rm2 = (rx * rx + ry * ry) + rz * rz;
      REAL thr = aa_create;
      if (rad) {
        /* a gap below -(r_i + r_j) bonds nothing (squaring would bond again) */
        double s = (double)rad[idx] + (double)rad[jdx] + gap;
        thr = s > 0.0 ? (REAL)(s * s) : (REAL)0;
      }
      if (rm2 < thr && rm2 > 1e-18) {
        inv_L0[kdx] = RSQRT_RN(rm2);
        ILtype[kdx] = 1;
      } else {
        ILtype[kdx] = 0;
      }
      for (int d = 0; d < 3; ++d) {
        Rij[3 * kdx + d] = 0;
        Oijt[3 * kdx + d] = 0;
        Mijn[3 * kdx + d] = 0;
        Mijt[3 * kdx + d] = 0;
      }
    }
  }
}

/* Fq/Mq non-null: order-independent sums.  Each slot's force (normal plus
 * shear) and moment ((twisting plus bending) plus the unsymmetric shear
 * moment) is rounded to fixed point (FIXQ) and added to the particle's 64-bit
 * accumulators, instead of the reference's running float sum over the slots.
 * These are the per-pair values and the exact sums of the engine's
 * deterministic mode; every per-slot quantity is the reference's. */
static void FN(forces_bpm_body)(const REAL* R, const REAL* V, const REAL* W, uint32_t N, const uint32_t* IL,
                                uint32_t* ILtype, const REAL* inv_L0, REAL* Rij, REAL* Oijt, REAL* Mijn,
                                REAL* Mijt, REAL* F, REAL* M, uint32_t IonP, REAL dt, REAL E, REAL G,
                                REAL b_r0, REAL Ec0, REAL Gc0, const REAL* slot_br, const REAL* slot_sn,
                                const REAL* slot_st, REAL* Fabs, REAL* Mabs, REAL* Fsens, int nobreak,
                                int64_t* Fq, int64_t* Mq) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL fs[3] = {0, 0, 0}, ms[3] = {0, 0, 0};
    int64_t fq[3] = {0, 0, 0}, mq[3] = {0, 0, 0};
    REAL fa[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
    double fsens = 0;
    const REAL Wi[3] = {W[idx], W[idx + N], W[idx + 2 * N]};
    const REAL Vi[3] = {V[idx], V[idx + N], V[idx + 2 * N]};
    for (uint32_t k = 0; k < IonP; ++k) {
      uint64_t kdx = (uint64_t)idx * IonP + k;
      uint32_t jdx = IL[kdx];
      if (jdx == ORC_EMPTY || ILtype[kdx] != 1) continue;
      const REAL b_r = slot_br ? slot_br[kdx] : b_r0;
      const REAL Ec = slot_sn ? slot_sn[kdx] : Ec0;
      const REAL Gc = slot_st ? slot_st[kdx] : Gc0;
      const REAL Wj[3] = {W[jdx], W[jdx + N], W[jdx + 2 * N]};
      const REAL Vj[3] = {V[jdx], V[jdx + N], V[jdx + 2 * N]};
      REAL* Rk = Rij + 3 * kdx;
      REAL* Ok = Oijt + 3 * kdx;
      REAL* Nk = Mijn + 3 * kdx;
      REAL* Tk = Mijt + 3 * kdx;
      const REAL il = inv_L0[kdx];
      /* dd_Calculate_rijm_nij_2, dem3.cu:41-55 */
      REAL rx = R[jdx] - R[idx], ry = R[jdx + N] - R[idx + N], rz = R[jdx + 2 * N] - R[idx + 2 * N];
      REAL rijm = NORM3(rx, ry, rz);
      REAL rinv = ONE / rijm;
      REAL n[3] = {rx * rinv, ry * rinv, rz * rinv};
      /* dd_Calculate_fijn_bpm_2, dem3.cu:94-106.  The reference's operation
       * order; the products fused into their sums here (FMA, one rounding) are
       * the ones the CUDA product fuses, so the two agree bit for bit. */
      REAL cef = E * (rijm - ONE / il) * il;
      REAL Sc = cef;
      cef *= b_r * b_r * PI;
      REAL fn[3] = {n[0] * cef, n[1] * cef, n[2] * cef};
      for (int d = 0; d < 3; ++d) fs[d] += fn[d];
      /* dd_Calculate_M123_bpm_2, dem3.cu:57-92 */
      REAL tmp[3] = {FMA(Rk[1], n[2], -(Rk[2] * n[1])), FMA(Rk[2], n[0], -(Rk[0] * n[2])),
                     FMA(Rk[0], n[1], -(Rk[1] * n[0]))};
      cef = FMA(Wj[2] + Wi[2], n[2], FMA(Wj[1] + Wi[1], n[1], (Wj[0] + Wi[0]) * n[0])) * dt * HALF;
      REAL phi[3] = {n[0] * cef, n[1] * cef, n[2] * cef};
      Rk[0] = n[0];
      Rk[1] = n[1];
      Rk[2] = n[2];
      REAL M1[3], M2[3], M3[3];
      M1[0] = FMA(tmp[1], phi[1], FMA(tmp[2], phi[2], ONE));
      M1[1] = FMA(-tmp[1], phi[0], phi[2] - tmp[2]);
      M1[2] = FMA(-tmp[2], phi[0], -phi[1]) + tmp[1];
      M2[0] = FMA(-tmp[0], phi[1], tmp[2] - phi[2]);
      M2[1] = FMA(tmp[0], phi[0], FMA(tmp[2], phi[2], ONE));
      M2[2] = FMA(-tmp[2], phi[1], phi[0]) - tmp[0];
      M3[0] = FMA(-tmp[0], phi[2], -tmp[1]) + phi[1];
      M3[1] = FMA(-tmp[1], phi[2], tmp[0]) - phi[0];
      M3[2] = FMA(tmp[0], phi[0], tmp[1] * phi[1]) + ONE;
      /* dd_Calculate_mijn_bpm_2, dem3.cu:108-132 */
      const REAL dw[3] = {Wj[0] - Wi[0], Wj[1] - Wi[1], Wj[2] - Wi[2]};
      const REAL wn = FMA(n[2], dw[2], FMA(n[1], dw[1], n[0] * dw[0]));
      REAL cef1 = wn * (dt * HALF * G * il);
      REAL mn[3];
      mn[0] = FMA(n[0], cef1, FMA(M1[2], Nk[2], FMA(M1[1], Nk[1], M1[0] * Nk[0])));
      mn[1] = FMA(n[1], cef1, FMA(M2[2], Nk[2], FMA(M2[1], Nk[1], M2[0] * Nk[0])));
      mn[2] = FMA(n[2], cef1, FMA(M3[2], Nk[2], FMA(M3[1], Nk[1], M3[0] * Nk[0])));
      Nk[0] = mn[0];
      Nk[1] = mn[1];
      Nk[2] = mn[2];
      cef1 = PI * b_r * b_r * b_r * b_r;
      REAL tn[3] = {mn[0] * cef1, mn[1] * cef1, mn[2] * cef1};
      for (int d = 0; d < 3; ++d) ms[d] += tn[d];
      /* dd_Calculate_mijt_bpm_2, dem3.cu:134-155 */
      REAL cef2 = dt * QUARTER * E * il;
      REAL mt[3];
      mt[0] = FMA(FMA(-n[0], wn, dw[0]), cef2, FMA(M1[2], Tk[2], FMA(M1[1], Tk[1], M1[0] * Tk[0])));
      mt[1] = FMA(FMA(-n[1], wn, dw[1]), cef2, FMA(M2[2], Tk[2], FMA(M2[1], Tk[1], M2[0] * Tk[0])));
      mt[2] = FMA(FMA(-n[2], wn, dw[2]), cef2, FMA(M3[2], Tk[2], FMA(M3[1], Tk[1], M3[0] * Tk[0])));
      Tk[0] = mt[0];
      Tk[1] = mt[1];
      Tk[2] = mt[2];
      cef2 *= PI * b_r * b_r * b_r * b_r;
      REAL tt[3] = {mt[0] * cef2, mt[1] * cef2, mt[2] * cef2};
      for (int d = 0; d < 3; ++d) ms[d] += tt[d];
      /* dd_Calculate_fijt_mijunsym_bpm_2, dem3.cu:157-200 */
      REAL wsd[3] = {HALF * (Wj[0] + Wi[0]), HALF * (Wj[1] + Wi[1]), HALF * (Wj[2] + Wi[2])};
      REAL vij[3];
      vij[0] = FMA(wsd[2], ry, FMA(-wsd[1], rz, Vj[0] - Vi[0]));
      vij[1] = FMA(wsd[0], rz, FMA(-wsd[2], rx, Vj[1] - Vi[1]));
      vij[2] = FMA(wsd[1], rx, FMA(-wsd[0], ry, Vj[2] - Vi[2]));
      cef = FMA(n[2], vij[2], FMA(n[1], vij[1], n[0] * vij[0]));
      REAL ot[3];
      ot[0] = FMA(FMA(-n[0], cef, vij[0]), dt, FMA(M1[2], Ok[2], FMA(M1[1], Ok[1], M1[0] * Ok[0])));
      ot[1] = FMA(FMA(-n[1], cef, vij[1]), dt, FMA(M2[2], Ok[2], FMA(M2[1], Ok[1], M2[0] * Ok[0])));
      ot[2] = FMA(FMA(-n[2], cef, vij[2]), dt, FMA(M3[2], Ok[2], FMA(M3[1], Ok[1], M3[0] * Ok[0])));
      cef = G * il;
      REAL Mc = cef;
      cef *= b_r * b_r * PI;
      REAL ft[3] = {ot[0] * cef, ot[1] * cef, ot[2] * cef};
      for (int d = 0; d < 3; ++d) fs[d] += ft[d];
      Ok[0] = ot[0];
      Ok[1] = ot[1];
      Ok[2] = ot[2];
      REAL mu[3];
      mu[0] = HALF * FMA(ry, ot[2], -(rz * ot[1])) * cef;
      mu[1] = HALF * FMA(rz, ot[0], -(rx * ot[2])) * cef;
      mu[2] = HALF * FMA(rx, ot[1], -(ry * ot[0])) * cef;
      for (int d = 0; d < 3; ++d) ms[d] += mu[d];
      if (Fq)
        for (int d = 0; d < 3; ++d) {
          fq[d] += FIXQ(fn[d] + ft[d]);
          mq[d] += FIXQ((tn[d] + tt[d]) + mu[d]);
        }
      if (Fabs)
        for (int d = 0; d < 3; ++d) fa[d] += FABS(fn[d]) + FABS(ft[d]);
      if (Mabs)
        for (int d = 0; d < 3; ++d) ma[d] += FABS(tn[d]) + FABS(tt[d]) + FABS(mu[d]);
      /* normal stiffness times one ulp of the pair distance */
      if (Fsens) fsens += (double)(E * (b_r * b_r * PI) * il) * (double)ULP(rijm);
      /* dd_CheckBreakConditionDEM_2, dem3.cu:20-39 */
      if (!nobreak) {
        /* history norms: sqrt(z*z + (y*y + x*x)) with fused sums (the
         * reference's norm3df is not correctly rounded either) */
        Mc *= SQRT(FMA(Ok[2], Ok[2], FMA(Ok[1], Ok[1], Ok[0] * Ok[0])));
        Sc += SQRT(FMA(Tk[2], Tk[2], FMA(Tk[1], Tk[1], Tk[0] * Tk[0]))) * FOUR * b_r;
        Mc += SQRT(FMA(Nk[2], Nk[2], FMA(Nk[1], Nk[1], Nk[0] * Nk[0]))) * TWO * b_r;
        if ((Sc > Ec) || (Mc > Gc)) {
          ILtype[kdx] = 0;
          for (int d = 0; d < 3; ++d) {
            Ok[d] = 0;
            Nk[d] = 0;
            Tk[d] = 0;
          }
        }
      }
    }
    if (Fq) {
      for (int d = 0; d < 3; ++d) {
        Fq[idx + (size_t)d * N] += fq[d];
        Mq[idx + (size_t)d * N] += mq[d];
      }
    } else {
      F[idx] += fs[0];
      F[idx + N] += fs[1];
      F[idx + 2 * N] += fs[2];
      M[idx] += ms[0];
      M[idx + N] += ms[1];
      M[idx + 2 * N] += ms[2];
    }
    if (Fabs) {
      Fabs[idx] += fa[0];
      Fabs[idx + N] += fa[1];
      Fabs[idx + 2 * N] += fa[2];
    }
    if (Mabs) {
      Mabs[idx] += ma[0];
      Mabs[idx + N] += ma[1];
      Mabs[idx + 2 * N] += ma[2];
    }
    if (Fsens) Fsens[idx] += (REAL)fsens;
  }
}

/* Fq/Mq non-null: as forces_bpm_body, per contact the force (normal plus
 * tangential) and the moment (tangential plus rolling) in fixed point. */
static void FN(forces_hm_body)(const REAL* R, const REAL* V, const REAL* W, uint32_t N, const uint32_t* IL,
                               const uint32_t* ILtype, REAL* Oijt, REAL* F, REAL* M, uint32_t IonP, REAL dt,
                               REAL hmE, REAL hmG, REAL pA, REAL mu, REAL mur, REAL mP, REAL rP,
                               const REAL* rad, const REAL* mass, REAL* Fabs, REAL* Mabs, REAL* Fsens,
                               int64_t* Fq, int64_t* Mq) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL fs[3] = {0, 0, 0}, ms[3] = {0, 0, 0};
    int64_t fq[3] = {0, 0, 0}, mq[3] = {0, 0, 0};
    REAL fa[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
    double fsens = 0;
    int any_touch = 0;
    const REAL Wi[3] = {W[idx], W[idx + N], W[idx + 2 * N]};
    const REAL Vi[3] = {V[idx], V[idx + N], V[idx + 2 * N]};
    const REAL wim = (Wi[0] * Wi[0] + Wi[1] * Wi[1]) + Wi[2] * Wi[2];
    for (uint32_t k = 0; k < IonP; ++k) {
      uint64_t kdx = (uint64_t)idx * IonP + k;
      uint32_t jdx = IL[kdx];
      REAL* Ok = Oijt + 3 * kdx;
      if (jdx == ORC_EMPTY) {
        Ok[0] = 0;
        Ok[1] = 0;
        Ok[2] = 0;
        continue;
      }
      if (ILtype[kdx] != 0) continue;
      REAL rx = R[jdx] - R[idx], ry = R[jdx + N] - R[idx + N], rz = R[jdx + 2 * N] - R[idx + 2 * N];
      REAL rijm = NORM3(rx, ry, rz);
      REAL rinv = ONE / rijm;
      REAL n[3] = {rx * rinv, ry * rinv, rz * rinv};
      const REAL ri = rad ? rad[idx] : rP, rj = rad ? rad[jdx] : rP;
      const REAL sumr = rad ? ri + rj : TWO * rP;
      if (!(rijm < sumr)) {
        Ok[0] = 0;
        Ok[1] = 0;
        Ok[2] = 0;
        continue;
      }
      any_touch = 1;
      const REAL Wj[3] = {W[jdx], W[jdx + N], W[jdx + 2 * N]};
      const REAL Vj[3] = {V[jdx], V[jdx + N], V[jdx + 2 * N]};
      /* dd_Calculate_fijn_ppHM_2, dem3.cu:202-256 */
      REAL cef1, Kn, Kt, vij[3], m2;
      if (!rad) {
        cef1 = SQRT(rP * FABS(rP - HALF * rijm));
        vij[0] = Vj[0] - Vi[0] + rP * (n[1] * (Wj[2] + Wi[2]) - n[2] * (Wj[1] + Wi[1]));
        vij[1] = Vj[1] - Vi[1] + rP * (n[2] * (Wj[0] + Wi[0]) - n[0] * (Wj[2] + Wi[2]));
        vij[2] = Vj[2] - Vi[2] + rP * (n[0] * (Wj[1] + Wi[1]) - n[1] * (Wj[0] + Wi[0]));
        m2 = mP;
      } else {
        /* polydisperse generalisation: R* = r_i r_j/(r_i+r_j), overlap r_i+r_j-r,
         * contact velocity Vj-Vi + r_i n x Wi + r_j n x Wj, m* = m_i m_j/(m_i+m_j)
         * carried as 2 m* = m_a * (2 m_b/(m_a+m_b)), m_a the smaller mass, so
         * equal masses give m_i and both slots of the pair the same value. */
        REAL reff = ri * rj / sumr;
        cef1 = SQRT(reff * (sumr - rijm));
        REAL rbar = HALF * sumr, rdif = HALF * (rj - ri);
        REAL sw[3] = {Wj[0] + Wi[0], Wj[1] + Wi[1], Wj[2] + Wi[2]};
        REAL dw[3] = {Wj[0] - Wi[0], Wj[1] - Wi[1], Wj[2] - Wi[2]};
        vij[0] = Vj[0] - Vi[0] + rbar * (n[1] * sw[2] - n[2] * sw[1]) + rdif * (n[1] * dw[2] - n[2] * dw[1]);
        vij[1] = Vj[1] - Vi[1] + rbar * (n[2] * sw[0] - n[0] * sw[2]) + rdif * (n[2] * dw[0] - n[0] * dw[2]);
        vij[2] = Vj[2] - Vi[2] + rbar * (n[0] * sw[1] - n[1] * sw[0]) + rdif * (n[0] * dw[1] - n[1] * dw[0]);
        REAL mi = mass[idx], mj = mass[jdx];
        REAL ma = mi < mj ? mi : mj, mb = mi < mj ? mj : mi; /* symmetric in the pair */
        m2 = ma * ((mb + mb) / (ma + mb));
      }
      Kn = TWO * hmE * cef1;
      Kt = EIGHT * hmG * cef1;
      REAL vn = n[0] * vij[0] + n[1] * vij[1] + n[2] * vij[2];
      REAL fijnm = (rijm - sumr) * Kn * TWO_THIRDS;
      cef1 = DAMP * pA * vn * SQRT(Kn * HALF * m2);
      REAL fnv[3] = {n[0] * (fijnm + cef1), n[1] * (fijnm + cef1), n[2] * (fijnm + cef1)};
      for (int d = 0; d < 3; ++d) fs[d] += fnv[d];
      REAL vt[3] = {vij[0] - n[0] * vn, vij[1] - n[1] * vn, vij[2] - n[2] * vn};
      /* dd_Calculate_fijtmijt_ppHM_2, dem3.cu:258-317 */
      REAL ot[3];
      cef1 = n[0] * Ok[0] + n[1] * Ok[1] + n[2] * Ok[2];
      ot[0] = Ok[0] - n[0] * cef1;
      ot[1] = Ok[1] - n[1] * cef1;
      ot[2] = Ok[2] - n[2] * cef1;
      cef1 = (ot[0] * ot[0] + ot[1] * ot[1]) + ot[2] * ot[2];
      if (cef1 > 1e-18) {
        cef1 = ONE / cef1;
        cef1 *= (Ok[0] * Ok[0] + Ok[1] * Ok[1]) + Ok[2] * Ok[2];
        cef1 = SQRT(cef1);
        ot[0] *= cef1;
        ot[1] *= cef1;
        ot[2] *= cef1;
      }
      ot[0] += vt[0] * dt;
      ot[1] += vt[1] * dt;
      ot[2] += vt[2] * dt;
      REAL ft[3] = {ot[0] * Kt, ot[1] * Kt, ot[2] * Kt};
      REAL ftmm = (ft[0] * ft[0] + ft[1] * ft[1]) + ft[2] * ft[2];
      if (ftmm > mu * mu * fijnm * fijnm) {
        cef1 = mu * FABS(fijnm) * RSQRT_RN(ftmm);
        ft[0] *= cef1;
        ft[1] *= cef1;
        ft[2] *= cef1;
        cef1 = ONE / Kt;
        ot[0] = ft[0] * cef1;
        ot[1] = ft[1] * cef1;
        ot[2] = ft[2] * cef1;
      } else {
        cef1 = DAMP * pA * SQRT(Kt * HALF * m2);
        ft[0] += vt[0] * cef1;
        ft[1] += vt[1] * cef1;
        ft[2] += vt[2] * cef1;
      }
      Ok[0] = ot[0];
      Ok[1] = ot[1];
      Ok[2] = ot[2];
      for (int d = 0; d < 3; ++d) fs[d] += ft[d];
      REAL mt[3] = {(n[1] * ft[2] - n[2] * ft[1]) * ri, (n[2] * ft[0] - n[0] * ft[2]) * ri,
                    (n[0] * ft[1] - n[1] * ft[0]) * ri};
      for (int d = 0; d < 3; ++d) ms[d] += mt[d];
      /* dd_Calculate_mijroll_ppHM_2, dem3.cu:319-339 */
      REAL mr[3] = {0, 0, 0};
      if (wim > 1e-18) {
        cef1 = -mur * FABS(fijnm) * RSQRT_RN(wim);
        mr[0] = Wi[0] * cef1;
        mr[1] = Wi[1] * cef1;
        mr[2] = Wi[2] * cef1;
        for (int d = 0; d < 3; ++d) ms[d] += mr[d];
      }
      if (Fq)
        for (int d = 0; d < 3; ++d) {
          fq[d] += FIXQ(fnv[d] + ft[d]);
          mq[d] += FIXQ(mt[d] + mr[d]);
        }
      if (Fabs)
        for (int d = 0; d < 3; ++d) fa[d] += FABS(fnv[d]) + FABS(ft[d]);
      if (Mabs)
        for (int d = 0; d < 3; ++d) ma[d] += FABS(mt[d]) + FABS(mr[d]);
      if (Fsens) fsens += (double)Kn * (double)ULP(rijm);
    }
    /* The reference's else-branch of dd_Calculate_mijroll_ppHM_2 clears the
     * whole accumulated contact moment of the particle whenever |w_i|^2 <= 1e-18;
     * since that test does not change along the slot loop, the particle then
     * receives no contact moment at all this step. */
    if (any_touch && !(wim > 1e-18)) {
      ms[0] = 0;
      ms[1] = 0;
      ms[2] = 0;
      mq[0] = 0;
      mq[1] = 0;
      mq[2] = 0;
    }
    if (Fq) {
      for (int d = 0; d < 3; ++d) {
        Fq[idx + (size_t)d * N] += fq[d];
        Mq[idx + (size_t)d * N] += mq[d];
      }
    } else {
      F[idx] += fs[0];
      F[idx + N] += fs[1];
      F[idx + 2 * N] += fs[2];
      M[idx] += ms[0];
      M[idx + N] += ms[1];
      M[idx + 2 * N] += ms[2];
    }
    if (Fabs) {
      Fabs[idx] += fa[0];
      Fabs[idx + N] += fa[1];
      Fabs[idx + 2 * N] += fa[2];
    }
    if (Mabs) {
      Mabs[idx] += ma[0];
      Mabs[idx + N] += ma[1];
      Mabs[idx + 2 * N] += ma[2];
    }
    if (Fsens) Fsens[idx] += (REAL)fsens;
  }
}

void FN(orc_forces_bpm)(const REAL* R, const REAL* V, const REAL* W, uint32_t N, const uint32_t* IL,
                        uint32_t* ILtype, const REAL* inv_L0, REAL* Rij, REAL* Oijt, REAL* Mijn,
                        REAL* Mijt, REAL* F, REAL* M, uint32_t IonP, REAL dt, REAL E, REAL G,
                        REAL b_r0, REAL Ec0, REAL Gc0, const REAL* slot_br, const REAL* slot_sn,
                        const REAL* slot_st, REAL* Fabs, REAL* Mabs, REAL* Fsens, int nobreak) {
  FN(forces_bpm_body)(R, V, W, N, IL, ILtype, inv_L0, Rij, Oijt, Mijn, Mijt, F, M, IonP, dt, E, G, b_r0, Ec0,
                      Gc0, slot_br, slot_sn, slot_st, Fabs, Mabs, Fsens, nobreak, NULL, NULL);
}

void FN(orc_forces_bpm_q)(const REAL* R, const REAL* V, const REAL* W, uint32_t N, const uint32_t* IL,
                          uint32_t* ILtype, const REAL* inv_L0, REAL* Rij, REAL* Oijt, REAL* Mijn,
                          REAL* Mijt, uint32_t IonP, REAL dt, REAL E, REAL G, REAL b_r0, REAL Ec0,
                          REAL Gc0, const REAL* slot_br, const REAL* slot_sn, const REAL* slot_st,
                          int nobreak, int64_t* Fq, int64_t* Mq) {
  FN(forces_bpm_body)(R, V, W, N, IL, ILtype, inv_L0, Rij, Oijt, Mijn, Mijt, NULL, NULL, IonP, dt, E, G, b_r0,
                      Ec0, Gc0, slot_br, slot_sn, slot_st, NULL, NULL, NULL, nobreak, Fq, Mq);
}

void FN(orc_forces_hm)(const REAL* R, const REAL* V, const REAL* W, uint32_t N, const uint32_t* IL,
                       const uint32_t* ILtype, REAL* Oijt, REAL* F, REAL* M, uint32_t IonP, REAL dt,
                       REAL hmE, REAL hmG, REAL pA, REAL mu, REAL mur, REAL mP, REAL rP,
                       const REAL* rad, const REAL* mass, REAL* Fabs, REAL* Mabs, REAL* Fsens) {
  FN(forces_hm_body)(R, V, W, N, IL, ILtype, Oijt, F, M, IonP, dt, hmE, hmG, pA, mu, mur, mP, rP, rad, mass,
                     Fabs, Mabs, Fsens, NULL, NULL);
}

void FN(orc_forces_hm_q)(const REAL* R, const REAL* V, const REAL* W, uint32_t N, const uint32_t* IL,
                         const uint32_t* ILtype, REAL* Oijt, uint32_t IonP, REAL dt, REAL hmE, REAL hmG,
                         REAL pA, REAL mu, REAL mur, REAL mP, REAL rP, const REAL* rad, const REAL* mass,
                         int64_t* Fq, int64_t* Mq) {
  FN(forces_hm_body)(R, V, W, N, IL, ILtype, Oijt, NULL, NULL, IonP, dt, hmE, hmG, pA, mu, mur, mP, rP, rad,
                     mass, NULL, NULL, NULL, Fq, Mq);
}

/* F = the fixed-point sums converted back (UNFIXQ), one value per element */
void FN(orc_fix_to_real)(const int64_t* q, REAL* out, uint64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)n; ++k) out[k] = UNFIXQ(q[k]);
}

/* one particle-platen contact, md_compression_hm.cu:20-154 ; returns the
 * normal force component along the platen axis */
static inline REAL FN(wall_contact)(int axis, REAL sgn, const REAL* V, const REAL* W, REAL* Oiwt,
                                    REAL* F, REAL* M, uint32_t N, uint32_t idx, REAL dt, REAL wE,
                                    REAL wG, REAL pA, REAL mu, REAL mur, REAL mP, REAL rP, REAL riwm,
                                    REAL wallvel) {
  REAL niw[3] = {0, 0, 0}, wallv[3] = {0, 0, 0};
  niw[axis] = sgn;
  wallv[axis] = wallvel;
  const REAL Wi[3] = {W[idx], W[idx + N], W[idx + 2 * N]};
  const REAL Vi[3] = {V[idx], V[idx + N], V[idx + 2 * N]};
  /* dd_Calculate_fijn_pwHM_2 */
  REAL cef1 = SQRT(rP * FABS(rP - riwm));
  REAL Kn = TWO * wE * cef1;
  REAL Kt = EIGHT * wG * cef1;
  REAL viw[3];
  viw[0] = wallv[0] - Vi[0] + rP * (niw[1] * Wi[2] - niw[2] * Wi[1]);
  viw[1] = wallv[1] - Vi[1] + rP * (niw[2] * Wi[0] - niw[0] * Wi[2]);
  viw[2] = wallv[2] - Vi[2] + rP * (niw[0] * Wi[1] - niw[1] * Wi[0]);
  REAL vn = niw[0] * viw[0] + niw[1] * viw[1] + niw[2] * viw[2];
  REAL fiwnm = (riwm - rP) * Kn * TWO_THIRDS;
  cef1 = DAMP * pA * vn * SQRT(Kn * mP);
  REAL fiwn[3] = {niw[0] * (fiwnm + cef1), niw[1] * (fiwnm + cef1), niw[2] * (fiwnm + cef1)};
  REAL vt[3] = {viw[0] - niw[0] * vn, viw[1] - niw[1] * vn, viw[2] - niw[2] * vn};
  /* dd_Calculate_fijtmijt_pwHM_2 */
  REAL o_[3] = {Oiwt[idx], Oiwt[idx + N], Oiwt[idx + 2 * N]};
  cef1 = niw[0] * o_[0] + niw[1] * o_[1] + niw[2] * o_[2];
  REAL ot[3] = {o_[0] - niw[0] * cef1, o_[1] - niw[1] * cef1, o_[2] - niw[2] * cef1};
  cef1 = (ot[0] * ot[0] + ot[1] * ot[1]) + ot[2] * ot[2];
  if (cef1 > 1e-18) {
    cef1 = ONE / cef1;
    /* md_compression_hm.cu:91 multiplies x by y in the first term */
    cef1 *= (o_[0] * o_[1] + o_[1] * o_[1]) + o_[2] * o_[2];
    cef1 = SQRT(cef1);
    ot[0] *= cef1;
    ot[1] *= cef1;
    ot[2] *= cef1;
  }
  ot[0] += vt[0] * dt;
  ot[1] += vt[1] * dt;
  ot[2] += vt[2] * dt;
  REAL ft[3] = {ot[0] * Kt, ot[1] * Kt, ot[2] * Kt};
  REAL ftmm = (ft[0] * ft[0] + ft[1] * ft[1]) + ft[2] * ft[2];
  if (ftmm > mu * mu * fiwnm * fiwnm) {
    cef1 = mu * FABS(fiwnm) * RSQRT_RN(ftmm);
    ft[0] *= cef1;
    ft[1] *= cef1;
    ft[2] *= cef1;
    cef1 = ONE / Kt;
    ot[0] = ft[0] * cef1;
    ot[1] = ft[1] * cef1;
    ot[2] = ft[2] * cef1;
  } else {
    cef1 = DAMP * pA * SQRT(Kt * mP);
    ft[0] += vt[0] * cef1;
    ft[1] += vt[1] * cef1;
    ft[2] += vt[2] * cef1;
  }
  Oiwt[idx] = ot[0];
  Oiwt[idx + N] = ot[1];
  Oiwt[idx + 2 * N] = ot[2];
  REAL mt[3] = {(niw[1] * ft[2] - niw[2] * ft[1]) * rP, (niw[2] * ft[0] - niw[0] * ft[2]) * rP,
                (niw[0] * ft[1] - niw[1] * ft[0]) * rP};
  REAL wim = (Wi[0] * Wi[0] + Wi[1] * Wi[1]) + Wi[2] * Wi[2];
  REAL madd[3] = {0, 0, 0};
  if (wim > 1e-18) {
    cef1 = -mur * FABS(fiwnm) * RSQRT_RN(wim);
    madd[0] = Wi[0] * cef1;
    madd[1] = Wi[1] * cef1;
    madd[2] = Wi[2] * cef1;
  }
  F[idx] += fiwn[0] + ft[0];
  F[idx + N] += fiwn[1] + ft[1];
  F[idx + 2 * N] += fiwn[2] + ft[2];
  M[idx] += mt[0] + madd[0];
  M[idx + N] += mt[1] + madd[1];
  M[idx + 2 * N] += mt[2] + madd[2];
  return fiwn[axis];
}

static void FN(platen_body)(int axis, const REAL* R, const REAL* V, const REAL* W, REAL* Oiwt, REAL* F,
                           REAL* M, uint32_t N, REAL dt, REAL wE, REAL wG, REAL pA, REAL mu, REAL mur,
                           REAL mP, REAL rP, const REAL* rad, const REAL* mass, const REAL* c,
                           REAL wall_RR, REAL wall_top, REAL wall_bot, REAL wall_V, REAL Zcut, REAL* FL,
                           double* sFL, int fixsum);

void FN(orc_platen)(int axis, const REAL* R, const REAL* V, const REAL* W, REAL* Oiwt, REAL* F, REAL* M,
                    uint32_t N, REAL dt, REAL wE, REAL wG, REAL pA, REAL mu, REAL mur, REAL mP, REAL rP,
                    const REAL* rad, const REAL* mass, const REAL* c, REAL wall_RR, REAL wall_top,
                    REAL wall_bot, REAL wall_V, REAL Zcut, REAL* FL, double* sFL) {
  FN(platen_body)(axis, R, V, W, Oiwt, F, M, N, dt, wE, wG, pA, mu, mur, mP, rP, rad, mass, c, wall_RR, wall_top,
                  wall_bot, wall_V, Zcut, FL, sFL, 0);
}

/* The platen step with sFL summed as the engine's deterministic mode does:
 * every sphere's normal platen force, widened to double, rounded to a
 * multiple of 2^-40 and added as an integer (exact, order-independent). */
void FN(orc_platen_q)(int axis, const REAL* R, const REAL* V, const REAL* W, REAL* Oiwt, REAL* F, REAL* M,
                      uint32_t N, REAL dt, REAL wE, REAL wG, REAL pA, REAL mu, REAL mur, REAL mP, REAL rP,
                      const REAL* rad, const REAL* mass, const REAL* c, REAL wall_RR, REAL wall_top,
                      REAL wall_bot, REAL wall_V, REAL Zcut, double* sFL) {
  FN(platen_body)(axis, R, V, W, Oiwt, F, M, N, dt, wE, wG, pA, mu, mur, mP, rP, rad, mass, c, wall_RR, wall_top,
                  wall_bot, wall_V, Zcut, NULL, sFL, 1);
}

static void FN(platen_body)(int axis, const REAL* R, const REAL* V, const REAL* W, REAL* Oiwt, REAL* F,
                           REAL* M, uint32_t N, REAL dt, REAL wE, REAL wG, REAL pA, REAL mu, REAL mur,
                           REAL mP, REAL rP, const REAL* rad, const REAL* mass, const REAL* c,
                           REAL wall_RR, REAL wall_top, REAL wall_bot, REAL wall_V, REAL Zcut, REAL* FL,
                           double* sFL, int fixsum) {
  const uint32_t B = N / 64 + 1; /* md_data_types.h:66-70 */
  REAL* contrib_b = (REAL*)calloc((size_t)B * 64, sizeof(REAL));
  REAL* contrib_t = (REAL*)calloc((size_t)B * 64, sizeof(REAL));
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL r[3];
    int lat0, lat1; /* lateral axes of the cylinder test */
    if (axis == 2) {
      r[0] = R[idx] - c[0];
      r[1] = R[idx + N] - c[1];
      r[2] = R[idx + 2 * N];
      lat0 = 0;
      lat1 = 1;
    } else {
      r[0] = R[idx] - c[0];
      r[1] = R[idx + N];
      r[2] = R[idx + 2 * N] - c[2];
      lat0 = 0;
      lat1 = 2;
    }
    if (!(r[lat0] * r[lat0] + r[lat1] * r[lat1] < wall_RR && r[2] < Zcut)) continue;
    REAL ri = rad ? rad[idx] : rP;
    REAL mi = rad ? mass[idx] : mP;
    REAL s_t = 0, s_b = 0;
    if (wall_top - r[axis] < ri) {
      REAL riwm = FABS(wall_top - r[axis]);
      s_t = FN(wall_contact)(axis, ONE, V, W, Oiwt, F, M, N, idx, dt, wE, wG, pA, mu, mur, mi, ri,
                             riwm, wall_V);
    } else {
      Oiwt[idx] = 0;
      Oiwt[idx + N] = 0;
      Oiwt[idx + 2 * N] = 0;
    }
    if (r[axis] - wall_bot < ri) {
      REAL riwm = FABS(wall_bot - r[axis]);
      s_b = FN(wall_contact)(axis, -ONE, V, W, Oiwt, F, M, N, idx, dt, wE, wG, pA, mu, mur, mi, ri,
                             riwm, -wall_V);
    } else {
      Oiwt[idx] = 0;
      Oiwt[idx + N] = 0;
      Oiwt[idx + 2 * N] = 0;
    }
    contrib_t[idx] = -s_t;
    contrib_b[idx] = -s_b;
  }
  if (fixsum) {
    int64_t qb = 0, qt = 0;
    for (uint32_t idx = 0; idx < N; ++idx) {
      qb += llrint((double)contrib_b[idx] * 0x1p40);
      qt += llrint((double)contrib_t[idx] * 0x1p40);
    }
    if (sFL) {
      sFL[0] = (double)qb * 0x1p-40;
      sFL[1] = (double)qt * 0x1p-40;
    }
    free(contrib_b);
    free(contrib_t);
    return;
  }
  /* 64-thread shared-memory tree of md_compression_hm.cu:243-300, then the
   * host double sum of md_results.cu:58-69 */
  double sb = 0, st = 0;
  for (uint32_t b = 0; b < B; ++b) {
    REAL xb[64], xt[64];
    for (int t = 0; t < 64; ++t) {
      xb[t] = contrib_b[(size_t)b * 64 + t];
      xt[t] = contrib_t[(size_t)b * 64 + t];
    }
    for (int off = 32; off >= 1; off >>= 1)
      for (int t = 0; t < off; ++t) {
        xb[t] = xb[t] + xb[t + off];
        xt[t] = xt[t] + xt[t + off];
      }
    if (FL) {
      FL[b] = xb[0];
      FL[b + B] = xt[0];
    }
    sb += (double)xb[0];
    st += (double)xt[0];
  }
  if (sFL) {
    sFL[0] = sb;
    sFL[1] = st;
  }
  free(contrib_b);
  free(contrib_t);
}

void FN(orc_increments)(const REAL* F, REAL* V, REAL* R, const REAL* M, REAL* W, uint32_t N, REAL dtm,
                        REAL dt, REAL dtI, const REAL* dtm_i, const REAL* dtI_i) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL am = dtm_i ? dtm_i[idx] : dtm;
    REAL aI = dtI_i ? dtI_i[idx] : dtI;
    for (int d = 0; d < 3; ++d) {
      size_t k = idx + (size_t)d * N;
      V[k] += F[k] * am;
      R[k] += V[k] * dt;
      W[k] += M[k] * aI;
    }
  }
}

void FN(orc_cut_restriction)(REAL* R, REAL* V, REAL* F, uint32_t N, const REAL* c, const REAL* s2,
                             const REAL* hp) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL dr[3] = {R[idx] - c[0], R[idx + N] - c[1], R[idx + 2 * N] - c[2]};
    int out = 0;
    for (int d = 0; d < 3; ++d) {
      if (dr[d] - s2[d] > 0) out = 1;
      if (dr[d] + s2[d] < 0) out = 1;
    }
    if (out) {
      for (int d = 0; d < 3; ++d) {
        R[idx + (size_t)d * N] = hp[d];
        V[idx + (size_t)d * N] = 0;
        F[idx + (size_t)d * N] = 0;
      }
    }
  }
}

void FN(orc_soft_forces)(const REAL* R, REAL* F, uint32_t N, const uint32_t* IL, REAL* Rijm,
                         uint32_t IonP, REAL D, REAL aa, const REAL* rad) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL fs[3] = {0, 0, 0};
    for (uint32_t k = 0; k < IonP; ++k) {
      uint64_t kdx = (uint64_t)idx * IonP + k;
      uint32_t jdx = IL[kdx];
      if (jdx == ORC_EMPTY) {
        if (Rijm) Rijm[kdx] = (REAL)1e10;
        continue;
      }
      REAL dr[3] = {R[jdx] - R[idx], R[jdx + N] - R[idx + N], R[jdx + 2 * N] - R[idx + 2 * N]};
      REAL rr = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
      if (Rijm) Rijm[kdx] = rr;
      REAL a2 = aa;
      if (rad) {
        REAL s = rad[idx] + rad[jdx];
        a2 = s * s;
      }
      if (rr < a2) {
        REAL aa_d_rr = a2 * (ONE / rr);
        REAL fm = (-D) * aa_d_rr;
        fs[0] += fm * dr[0];
        fs[1] += fm * dr[1];
        fs[2] += fm * dr[2];
      }
    }
    F[idx] = fs[0];
    F[idx + N] = fs[1];
    F[idx + 2 * N] = fs[2];
  }
}

void FN(orc_fire_increments)(const REAL* F, REAL* V, REAL* R, uint32_t N, REAL dtm, REAL dt, REAL alpha,
                             const REAL* dtm_i) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL am = dtm_i ? dtm_i[idx] : dtm;
    REAL f3[3] = {F[idx], F[idx + N], F[idx + 2 * N]};
    REAL v[3] = {f3[0] * am, f3[1] * am, f3[2] * am};
    REAL vv = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
    REAL f = (f3[0] * f3[0] + f3[1] * f3[1]) + f3[2] * f3[2];
    REAL vdf;
    if (f > (REAL)1e-12f)
      vdf = alpha * SQRT(vv * (ONE / f));
    else
      vdf = alpha * SQRT(vv) * (REAL)1e6;
    for (int d = 0; d < 3; ++d) {
      v[d] = (ONE - alpha) * v[d] + vdf * f3[d];
      V[idx + (size_t)d * N] = v[d];
      R[idx + (size_t)d * N] += v[d] * dt;
    }
  }
}

void FN(orc_fire_half_step_back)(const REAL* V, REAL* R, uint32_t N, REAL dt_d2) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii)
    for (int d = 0; d < 3; ++d) R[ii + (int64_t)d * N] -= V[ii + (int64_t)d * N] * dt_d2;
}

double FN(orc_fdotv)(const REAL* V, const REAL* F, uint32_t N) {
  const uint32_t B = N / 256 + 1; /* md_firerelaxation.cu:74 */
  REAL total = 0;                 /* Fire.FdotV is a float accumulated on the host */
  for (uint32_t b = 0; b < B; ++b) {
    REAL s[64];
    for (uint32_t t = 0; t < 64; ++t) {
      uint32_t idx = b * 256 + t;
      REAL acc = 0;
      int cnt = 0;
      if (idx + 3 * 64 < N)
        cnt = 4;
      else if (idx + 2 * 64 < N)
        cnt = 3;
      else if (idx + 64 < N)
        cnt = 2;
      else if (idx < N)
        cnt = 1;
      for (int q = 0; q < cnt; ++q) {
        uint32_t i = idx + q * 64;
        REAL term = (F[i] * V[i] + F[i + N] * V[i + N]) + F[i + 2 * N] * V[i + 2 * N];
        acc = (q == 0) ? term : acc + term;
      }
      s[t] = acc;
    }
    for (int off = 32; off >= 1; off >>= 1)
      for (int t = 0; t < off; ++t) s[t] = s[t] + s[t + off];
    total += (REAL)s[0];
  }
  return (double)total;
}

void FN(orc_increments_viscous)(const REAL* F, REAL* V, REAL* R, uint32_t N, REAL dtm, REAL dt, REAL vis,
                                const REAL* dtm_i) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    REAL am = dtm_i ? dtm_i[ii] : dtm;
    for (int d = 0; d < 3; ++d) {
      int64_t k = ii + (int64_t)d * N;
      V[k] += (F[k] - V[k] * vis) * am;
      R[k] += V[k] * dt;
    }
  }
}

void FN(orc_cylinder_restriction_z)(REAL* V, REAL* R, uint32_t N, const REAL* c, REAL R0, REAL H0,
                                    REAL HideZ) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)N; ++ii) {
    uint32_t idx = (uint32_t)ii;
    REAL dr[3] = {R[idx] - c[0], R[idx + N] - c[1], R[idx + 2 * N] - c[2]};
    REAL s[3] = {0, 0, 0};
    REAL rr = dr[0] * dr[0] + dr[1] * dr[1];
    if (dr[2] < HideZ - c[2]) {
      if (rr > R0 * R0) {
        rr = RSQRT_RN(rr);
        s[0] = dr[0] * (R0 * rr - ONE);
        s[1] = dr[1] * (R0 * rr - ONE);
        V[idx] *= -ONE;
        V[idx + N] *= -ONE;
      }
      if (dr[2] > H0) {
        s[2] = H0 - dr[2];
        V[idx + 2 * N] *= -ONE;
      }
      if (dr[2] < -H0) {
        s[2] = -H0 - dr[2];
        V[idx + 2 * N] *= -ONE;
      }
      R[idx] += s[0];
      R[idx + N] += s[1];
      R[idx + 2 * N] += s[2];
    }
  }
}

#undef NORM3
#undef FN
#undef CAT
#undef CAT2
