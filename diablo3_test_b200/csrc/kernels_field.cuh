// Fourier-space column step split by field: the default path of the column
// solve.
//
// The implicit y operators of u1, u2, u3 and every scalar are the same in
// every (kx, kz) column (the horizontal terms are explicit, for/channel.f90
// :108-153), and a field's explicit terms read the other fields only as they
// were at the start of the substep.  So every (field, column) pair is an
// independent task until the projection, which couples the three velocities
// and the pressure through rem_div_chan (:946-1023).  The column step
// therefore runs as two kernels:
//
//   k_field_solve   a block per (field, 8 adjacent columns), a warp per
//                   column: explicit RK terms (:29-249), cf for the next
//                   substep, the explicit Crank-Nicolson half (:468-514,
//                   :625-633), the pressure gradient, the wall rows and the
//                   factored implicit solve (:657-877); writes the solved
//                   velocity u* (the scalars' final value);
//   k_project_cols  a block per 8 columns, a warp per column: divergence of
//                   u*, the pressure-correction Poisson solve, the
//                   projection and cp += phi/h (:901-1023).
//
// Data path.  A column's rows lie one plane apart in HBM; adjacent columns are
// adjacent in memory.  A block therefore moves each array as an
// (Ny+2) x 8-column tile: cp.async copies of 16 bytes, four 128-byte row
// segments per warp instruction, into a two-stage shared-memory ring, so the
// next tile is in flight while the current one is consumed.  Each warp then
// reads its own column from the tile, a lane owning R consecutive rows
// (csolve's partition solver), and results leave through a third tile slot
// with the same coalesced pattern.  Tile slots are XOR-swizzled by the lane
// that owns the row, so the 32 lanes' 16-byte reads spread over all eight
// 16-byte bank groups.
#pragma once
#include "common.cuh"
#include "kernels_solve.cuh"
#include "kernels_solve2.cuh"


struct FieldArgs {
  SolveArgs s;
  const double* kc;    // implicit rows of this substep [kind][3][n] (see Solve2Args)
  const double* met;   // [MET_N][n]
  const double* fac;   // factored systems of this substep (k_factor), kinds 0..2+N_th
  int nf;              // 3 + N_th
  int mean_split;      // see Solve2Args::mean_split
  const double* prof;  // [2][n] U1(j), I(U1)(j)
  // k_column_step's scheduler: [0] status (1 = a wait gave up), [1] task
  // counter, [2 + g] velocity solves done in column group g
  int* sched;
  int need;            // solves a projection waits for (3)
  int lag;             // column groups between a group's solves and its projection
  long long max_spins; // bound of a projection's wait
};

namespace cfield {
using namespace csolve;

// tile slot of row j, column c: the XOR key is the owning lane (j / R)
template <int R>
DI int slot(int j, int c) { return j * FS_COLS + (c ^ ((j / R) & 7)); }

DI void cp16(void* s, const void* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g));
}
DI void cp8(void* s, const void* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g));
}
DI void commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> DI void wait_groups() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Issue the copies of one tile (rows [0, n), columns q0 .. q0+nvalid-1 of g,
// plane stride ps elements of ESZ bytes) and close the copy group.
// g == nullptr closes an empty group, so every step commits exactly one.
// Thread t copies column t % 8 of rows t / 8, t / 8 + 32, ...
template <int R, int ESZ>
DI void load_tile(void* tile, const void* g, size_t ps, int q0, int nvalid, int n, int tid) {
  if (g) {
    const int c = tid & 7;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(tile);
    if (c < nvalid) {
      const char* gp = (const char*)g + ((size_t)(tid >> 3) * ps + q0 + c) * ESZ;
      const size_t gstep = (size_t)32 * ps * ESZ;
      for (int j = tid >> 3; j < n; j += 32, gp += gstep) {
        const unsigned sa = sbase + (unsigned)(j * FS_COLS + (c ^ ((j / R) & 7))) * ESZ;
        if (ESZ == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gp));
        else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gp));
      }
    } else {
      for (int j = tid >> 3; j < n; j += 32) {
        char* sp = (char*)tile + (j * FS_COLS + (c ^ ((j / R) & 7))) * ESZ;
        if (ESZ == 16) *(double2*)sp = make_double2(0.0, 0.0);
        else *(float2*)sp = make_float2(0.f, 0.f);
      }
    }
  }
  commit();
}

// Store rows [j0, j1] of a double2 tile to g (columns q0 .. q0+nvalid-1).
// Rows below `jk` are taken from `keep_src` instead (rows a solve leaves as
// they were), when it is set.
template <int R>
DI void store_tile(const double2* tile, double2* g, size_t ps, int q0, int nvalid, int j0, int j1,
                   int tid, const double2* keep_src = nullptr, int jk = 0) {
  const int c = tid & 7;
  if (c >= nvalid) return;
  const size_t gstep = (size_t)32 * ps;
  int j = j0 + (tid >> 3);
  size_t o = (size_t)j * ps + q0 + c;
  for (; j <= j1; j += 32, o += gstep)
    g[o] = (keep_src && j < jk) ? __ldg(keep_src + o) : tile[j * FS_COLS + (c ^ ((j / R) & 7))];
}
}  // namespace cfield

// ---- k_field_solve -------------------------------------------------------------
enum { FT_OWN = 0, FT_ADD, FT_BUOY, FT_NL, FT_CFOLD, FT_P };
struct FTile {
  const void* src;
  int kind, f32;
  double coef;
};
#define FS_MAXTILES (5 + 2 * SOLVE_MAXTH)

// Shared memory of both kernels: a two-stage ring of (Ny+2) x FS_COLS complex
// doubles.  Results leave through the slot just consumed.
inline size_t field_smem_bytes(int n) { return (size_t)2 * n * FS_COLS * sizeof(double2); }

namespace cfield {
// The tiles field f reads, in the order its explicit terms use them: the
// nonlinear terms and couplings first, so that cf is complete when the
// field's own tile arrives and its registers turn into the right-hand side's.
DI int field_tiles(const SolveArgs& a, int f, FTile* tl) {
  const int th = f - 3;
  int ns = 0;
  if (a.nl64[f]) tl[ns++] = FTile{a.nl64[f], FT_NL, 0, 0.0};
  else tl[ns++] = FTile{a.nl32[f], FT_NL, 1, 0.0};
  if (f == 0 || f == 2) {
    if (a.roinvd != 0.0) tl[ns++] = FTile{a.cu_in[2 - f], FT_ADD, 0, f == 0 ? a.roinvd : -a.roinvd};
    const double g = f == 0 ? a.grav_x : a.grav_z;
    if (g != 0.0)
      for (int t = 0; t < a.nth; ++t) tl[ns++] = FTile{a.cth_in[t], FT_ADD, 0, g};
  } else if (f == 1) {
    if (a.grav_y != 0.0)
      for (int t = 0; t < a.nth; ++t) tl[ns++] = FTile{a.cth_in[t], FT_BUOY, 0, a.grav_y};
  } else {
    if (a.dthdx[th] != 0.0) tl[ns++] = FTile{a.cu_in[0], FT_ADD, 0, -a.dthdx[th]};
    if (a.dthdz[th] != 0.0) tl[ns++] = FTile{a.cu_in[2], FT_ADD, 0, -a.dthdz[th]};
  }
  tl[ns++] = FTile{f < 3 ? (const void*)a.cu_in[f] : (const void*)a.cth_in[th], FT_OWN, 0, 0.0};
  if (a.rk > 1) tl[ns++] = FTile{a.cf_in[f], FT_CFOLD, 0, 0.0};
  if (f < 3) tl[ns++] = FTile{a.cp_in, FT_P, 0, 0.0};
  return ns;
}
template <int R>
DI void load_ftile(void* slot, const FTile* t, size_t ps, int q0, int nvalid, int n, int tid) {
  if (t && t->f32) load_tile<R, 8>(slot, t->src, ps, q0, nvalid, n, tid);
  else load_tile<R, 16>(slot, t ? t->src : nullptr, ps, q0, nvalid, n, tid);
}
}  // namespace cfield

// Blocks per SM the register cap of k_column_step is set for: three fit in
// 80 registers without spills up to R = 4; beyond that the projection's
// Poisson rows and the solve spill under that cap, so two.
template <int R>
constexpr int fs_min_blocks() { return R <= 4 ? 3 : 2; }

// Blocks per SM the register cap of k_field_solve is set for: three fit in
// 80 registers without spills up to R = 6; at R = 9 the solve spills under
// that cap (0.545 against 0.477 ms per launch at 256 x 257 x 256), so two.
template <int R>
constexpr int fs_field_min_blocks() { return R <= 6 ? 3 : 2; }

// Persistent: block b takes tasks b, b + gridDim.x, ... (task t = field
// t % N_F of column group t / N_F).  The ring runs on across tasks: the last
// step of a task already copies the next task's first tile, so the tile is in
// flight while this task's solve and stores run.
template <int R>
__global__ void __launch_bounds__(FS_THREADS, fs_field_min_blocks<R>()) k_field_solve(const __grid_constant__ FieldArgs A) {
  using namespace cfield;
  extern __shared__ __align__(16) unsigned char fs_smem[];
  const SolveArgs& a = A.s;
  const int n = a.n, nyp = a.nyp;
  const int tsz = n * FS_COLS;
  double2* ring = reinterpret_cast<double2*>(fs_smem);
  const int nf = A.nf;
  const int ntask = ((a.ncol + FS_COLS - 1) / FS_COLS) * nf;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const size_t ps = (size_t)a.ncol;          // plane stride (the Fourier pitch is 2Nkz+1)
  const double2 z2 = make_double2(0.0, 0.0);
  const int j0 = lane * R;
  const double* met = A.met;
  int t = blockIdx.x;
  if (t >= ntask) return;
  FTile tl[FS_MAXTILES];
  int ns = field_tiles(a, t % nf, tl);
  int step = 0;
  {
    const int q0 = (t / nf) * FS_COLS;
    load_ftile<R>(ring, &tl[0], ps, q0, min(FS_COLS, a.ncol - q0), n, tid);
  }
  for (; t < ntask; t += gridDim.x) {
    const int f = t % nf;
    const int q0 = (t / nf) * FS_COLS;
    const int nvalid = min(FS_COLS, a.ncol - q0);
    const int q = min(q0 + w, a.ncol - 1);   // a warp past the last column works on a copy
    const int m = q / a.nk2, kq = q % a.nk2;
    const bool m00 = (q0 + w == 0);
    const double kxm = a.kx[m], kzq = a.kz[kq];
    const double k2s = kxm * kxm + kzq * kzq;
    const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
    // field kind: solve index f (0 u1, 1 u2, 2 u3, 3+n scalar n),
    // row-coefficient index (0 u1/u3, 1 u2, 2+n scalar n), explicit rows
    // [lo, hi], wall rows
    const int th = f - 3;
    const int kc_kind = f == 1 ? 1 : (f < 3 ? 0 : 2 + th);
    int lo, hi, b0, b1;
    double c0, c1;
    if (f == 0) { lo = a.jstart; hi = a.jend; b0 = a.ubc[0]; b1 = a.ubc[1]; c0 = a.uc1[0]; c1 = a.uc1[1]; }
    else if (f == 2) { lo = a.jstart; hi = a.jend; b0 = a.wbc[0]; b1 = a.wbc[1]; c0 = a.wc1[0]; c1 = a.wc1[1]; }
    else if (f == 1) { lo = 2; hi = nyp; b0 = a.vbc[0]; b1 = a.vbc[1]; c0 = a.vc1[0]; c1 = a.vc1[1]; }
    else { lo = a.jst[th]; hi = a.jet[th]; b0 = a.thbc[th][0]; b1 = a.thbc[th][1]; c0 = a.thc1[th][0]; c1 = a.thc1[th][1]; }
    const double* K = A.kc + (size_t)kc_kind * 3 * n;
    const double cfc = f >= 3 ? (a.nu / a.pr[th]) * kk : a.nu * kk;
    // mean-split correction of this field: -ikx U(j) u with U = U1 (u3,
    // scalars) or its GY interpolation I(U1) (u2); none for u1
    const double* Up = (A.mean_split && f != 0) ? A.prof + (f == 1 ? n : 0) : nullptr;
    const int tn = t + gridDim.x;

    double2 cr[R], cf[R];
#pragma unroll
    for (int r = 0; r < R; ++r) { cr[r] = z2; cf[r] = z2; }
    for (int k = 0; k < ns; ++k, ++step) {
      const FTile tk = tl[k];
      double2* nslot = ring + ((step + 1) & 1) * tsz;
      if (k + 1 < ns) {
        load_ftile<R>(nslot, &tl[k + 1], ps, q0, nvalid, n, tid);
      } else if (tn < ntask) {
        // the next task's first tile (its nonlinear terms)
        const int fn = tn % nf, qn = (tn / nf) * FS_COLS;
        const FTile first = a.nl64[fn] ? FTile{a.nl64[fn], FT_NL, 0, 0.0} : FTile{a.nl32[fn], FT_NL, 1, 0.0};
        load_ftile<R>(nslot, &first, ps, qn, min(FS_COLS, a.ncol - qn), n, tid);
      } else {
        load_ftile<R>(nslot, nullptr, ps, q0, nvalid, n, tid);
      }
      wait_groups<1>();
      __syncthreads();
      double2* T = ring + (step & 1) * tsz;
      auto TV = [&](int j) -> double2 { return T[slot<R>(j, w)]; };
      switch (tk.kind) {
        case FT_OWN: {
          // cf is complete here; it leaves through this slot, overwriting the
          // field row by row: a lane takes its two neighbour rows (other
          // lanes' rows of the same column) before the warp writes anything,
          // and reads row j+1 before overwriting row j
          // (lanes whose rows lie past the system read nothing)
          const double2 h_lo = (j0 >= 1 && j0 - 1 < n) ? TV(j0 - 1) : z2;
          const double2 h_hi = j0 + R < n ? TV(j0 + R) : z2;
          __syncwarp();
          double2 um = h_lo, u = j0 < n ? TV(j0) : z2;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            const double2 up = r == R - 1 ? h_hi : (j + 1 < n ? TV(j + 1) : z2);
            double2 c = cf[r];
            if (j >= lo && j <= hi) {
              c = c - cfc * u;
              if (Up) c = c - mul_ik(kxm * __ldg(Up + j), u);
              cr[r] = u - K[2 * n + j] * (up - u) + K[j] * (u - um);
              cr[r] = cr[r] + a.temp5 * c;
            }
            if (a.store_cf && j < n) T[slot<R>(j, w)] = c;
            um = u;
            u = up;
          }
          if (a.store_cf) {
            __syncthreads();
            store_tile<R>(T, a.cf_out[f], ps, q0, nvalid, lo, hi, tid);
          }
          break;
        }
        case FT_ADD:
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= lo && j <= hi) cf[r] = cf[r] + tk.coef * TV(j);
          }
          break;
        case FT_BUOY:
          if (!m00) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              if (j >= lo && j <= hi)
                cf[r] = cf[r] + tk.coef * (__ldg(met + MET_WB1 * n + j) * TV(j) +
                                           __ldg(met + MET_WB2 * n + j) * TV(j - 1));
            }
          }
          break;
        case FT_NL: {
          const float2* T32 = reinterpret_cast<const float2*>(T);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= lo && j <= hi) {
              double2 nl;
              if (tk.f32) { const float2 v = T32[slot<R>(j, w)]; nl = make_double2(v.x, v.y); }
              else nl = TV(j);
              cf[r] = -nl;
            }
          }
          break;
        }
        case FT_CFOLD:
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= lo && j <= hi) cr[r] = cr[r] + a.temp3 * TV(j);
          }
          break;
        case FT_P:
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= lo && j <= hi) {
              if (f == 0) {
                cr[r] = cr[r] - a.temp4 * mul_ik(kxm, TV(j));
                if (m00) cr[r].x -= a.px;
              } else if (f == 2) {
                cr[r] = cr[r] - a.temp4 * mul_ik(kzq, TV(j));
              } else {
                cr[r] = cr[r] - a.temp4 * __ldg(met + MET_IDY * n + j) * (TV(j) - TV(j - 1));
              }
            }
          }
          break;
        default:
          break;
      }
      __syncthreads();
    }
    // right-hand side: explicit terms on the explicit rows, wall values on
    // the wall rows (for/channel.f90:1545-1876); the matrix is in the factor
    // table
    const double v00 = m00 ? 1.0 : 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      double2 d = (j >= lo && j <= hi) ? cr[r] : z2;
      if (f == 1) {
        if (b0 == 0 && (j == 1 || j == 2)) d = make_double2(c0 * v00, 0);
        if (b0 == 1 && j == 1) d = make_double2(a.dyf[1] * c0 * v00, 0);
        if (j == 0) d = z2;
        if (b1 == 0 && (j == nyp || j == nyp + 1)) d = make_double2(c1 * v00, 0);
        if (b1 == 1 && j == nyp + 1) d = make_double2(a.dyf[nyp] * c1 * v00, 0);
      } else {
        if (j == 0 || j == nyp + 1) d = z2;
        if (j == 1) d = make_double2((b0 == 0 ? c0 : a.dy[2] * c0) * v00, 0);
        if (j == nyp) d = make_double2((b1 == 0 ? c1 : a.dy[nyp] * c1) * v00, 0);
      }
      cr[r] = d;
    }
    apply_factored<R>(A.fac + (size_t)f * Fac<R>::N * 32, cr, lane);
    // The solve writes rows w0 .. Ny+1 (u2: from row 1, the others from
    // lo - 1); rows below keep their input value.
    const int w0 = f == 1 ? 1 : lo - 1;
    double2* out = ring + ((step - 1) & 1) * tsz;   // the slot of the last step
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      if (j < n) out[slot<R>(j, w)] = cr[r];
    }
    __syncthreads();
    const double2* own = f < 3 ? a.cu_in[f] : a.cth_in[th];
    store_tile<R>(out, f < 3 ? a.cu_out[f] : a.cth_out[th], ps, q0, nvalid, 0, n - 1, tid, own, w0);
    __syncthreads();   // the next task's second tile goes to this slot
    if (tn < ntask) ns = field_tiles(a, tn % nf, tl);
  }
}

// ---- k_project_cols --------------------------------------------------------------
// Divergence -> pressure-correction Poisson solve -> projection -> pressure
// update, in place on cu_out (rem_div_chan, for/channel.f90:946-1023 with the
// wall rows of :1974-2015; cp_out = cp_in + phi/h, :905-911).  keep[q], if
// set, receives the velocity before the projection (the field courant reads,
// :885-888).  Tiles: u1*, u3*, u2* for the divergence; after the solve u1*,
// u3*, u2* again (from L2) and cp, each updated in its slot and stored.
// Persistent over column groups like k_field_solve.
template <int R>
__global__ void __launch_bounds__(FS_THREADS, 2) k_project_cols(const __grid_constant__ FieldArgs A) {
  using namespace cfield;
  extern __shared__ __align__(16) unsigned char fs_smem[];
  const SolveArgs& a = A.s;
  const int n = a.n, nyp = a.nyp;
  const int tsz = n * FS_COLS;
  double2* ring = reinterpret_cast<double2*>(fs_smem);
  const int ngroup = (a.ncol + FS_COLS - 1) / FS_COLS;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const size_t ps = (size_t)a.ncol;
  const double2 z2 = make_double2(0.0, 0.0);
  const int j0 = lane * R;
  const double* met = A.met;
  double2* const* cu = a.cu_out;
  const void* src[7] = {cu[0], cu[2], cu[1], cu[0], cu[2], cu[1], a.cp_in};
  const double ih = 1.0 / a.temp4;
  int g = blockIdx.x;
  if (g >= ngroup) return;
  load_tile<R, 16>(ring, src[0], ps, g * FS_COLS, min(FS_COLS, a.ncol - g * FS_COLS), n, tid);
  int step = 0;
  for (; g < ngroup; g += gridDim.x) {
    const int q0 = g * FS_COLS;
    const int nvalid = min(FS_COLS, a.ncol - q0);
    const int q = min(q0 + w, a.ncol - 1);
    const int m = q / a.nk2, kq = q % a.nk2;
    const bool m00 = (q0 + w == 0);
    const double kxm = a.kx[m], kzq = a.kz[kq];
    const int gn = g + gridDim.x;
    double2 d[R];
#pragma unroll
    for (int r = 0; r < R; ++r) d[r] = z2;
    double2 phm = z2;
    for (int k = 0; k < 7; ++k, ++step) {
      double2* nslot = ring + ((step + 1) & 1) * tsz;
      if (k + 1 < 7) load_tile<R, 16>(nslot, src[k + 1], ps, q0, nvalid, n, tid);
      else if (gn < ngroup) load_tile<R, 16>(nslot, src[0], ps, gn * FS_COLS, min(FS_COLS, a.ncol - gn * FS_COLS), n, tid);
      else load_tile<R, 16>(nslot, nullptr, ps, q0, nvalid, n, tid);
      wait_groups<1>();
      __syncthreads();
      double2* T = ring + (step & 1) * tsz;
      if (k < 3) {
        // divergence ik.u1 + ik.u3 + (u2(j+1) - u2(j))/dyf(j), rows 1..Ny,
        // in the order the solves of the fused step accumulated it
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= 1 && j <= nyp) {
            if (k == 0) d[r] = d[r] + mul_ik(kxm, T[slot<R>(j, w)]);
            else if (k == 1) d[r] = d[r] + mul_ik(kzq, T[slot<R>(j, w)]);
            else d[r] = d[r] + __ldg(met + MET_IDYF * n + j) * (T[slot<R>(j + 1, w)] - T[slot<R>(j, w)]);
          }
        }
        if (k == 2) {
          // Poisson rows: interior 1/(dy dyf) terms, Neumann walls, phi(1) = 0
          // for the (0,0) mode
          double al[R], cm[R];
          const double k2n = -kxm * kxm - kzq * kzq;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            double am = 0.0, cc = 0.0;
            if (j >= 1 && j <= nyp) { am = __ldg(met + MET_PA * n + j); cc = __ldg(met + MET_PC * n + j); }
            if (j == 1) { am = 0; cc = m00 ? 0.0 : -1.0; d[r] = z2; }
            if (j == nyp) { am = 1; cc = 0; d[r] = z2; }
            al[r] = am;
            cm[r] = cc;
          }
          csolve2::warp_tridiag_b<R>([&](int r) -> double& { return al[r]; }, [&](int r) -> double {
            const int j = j0 + r;
            return (j == 1) ? 1.0 : (j == nyp ? -1.0 : ((j > 1 && j < nyp) ? k2n + __ldg(met + MET_PB0 * n + j) : 1.0));
          }, [&](int r) -> double& { return cm[r]; }, d, lane);
          phm = shfl_up2(d[R - 1], 1);   // phi of the row below the lane's first
        }
      } else if (k < 6) {
        const int comp = k == 3 ? 0 : (k == 4 ? 2 : 1);
        if (a.keep[0]) {
          store_tile<R>(T, a.keep[comp], ps, q0, nvalid, 1, nyp, tid);
          __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (comp != 1 && j >= 1 && j <= nyp) {
            double2& u = T[slot<R>(j, w)];
            u = u - mul_ik(comp == 0 ? kxm : kzq, d[r]);
          }
          if (comp == 1 && j >= 2 && j <= nyp) {
            double2& u = T[slot<R>(j, w)];
            u = u - __ldg(met + MET_IDY * n + j) * (d[r] - (r == 0 ? phm : d[r - 1]));
          }
        }
        __syncthreads();
        store_tile<R>(T, cu[comp], ps, q0, nvalid, comp == 1 ? 2 : 1, nyp, tid);
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= a.jstart && j <= a.jend) {
            double2& p = T[slot<R>(j, w)];
            p = p + ih * d[r];
          }
        }
        __syncthreads();
        store_tile<R>(T, a.cp_out, ps, q0, nvalid, 0, n - 1, tid);
      }
      __syncthreads();
    }
  }
}

// ---- k_column_step --------------------------------------------------------------
// Both halves of the column step in one persistent launch.  Tasks are claimed
// in order from a counter: the field tasks of column group s (one per field)
// are followed, LAG groups later, by the projection task of group s - LAG, so
// the solved velocities it reads were written shortly before and are still
// in L2.  A projection task waits until its group's three velocity tasks have
// published their completion (a release/acquire count per group).  It can
// only wait on tasks claimed before it by blocks that are running, and field
// tasks never wait, so the wait always ends; it is still bounded by
// max_spins, after which the task sets the status word and leaves its group
// untouched, later waits give up at once, and the host reports
// DIABLO_ERR_TIMEOUT.
// Scheduler words: the status stays set across launches until the host has
// read it (a later launch's waits then give up at once); the task counter and
// the per-group counts are zeroed before every launch.
enum { SCHED_STATUS = 0, SCHED_COUNTER = 1, SCHED_DONE = 2 };

namespace cfield {
struct Task {
  int kind;   // 0 field solve, 1 projection, 2 none left
  int g, f;   // column group, field
  int mem;    // member (context) of the task
};
DI Task decode_task(int t, int ngroup, int nf, int lag) {
  const int a0 = lag * nf, a1 = a0 + (ngroup - lag) * (nf + 1), a2 = a1 + lag;
  if (t < a0) return Task{0, t / nf, t % nf, 0};
  if (t < a1) {
    const int u = t - a0, s = lag + u / (nf + 1), r = u % (nf + 1);
    return r < nf ? Task{0, s, r, 0} : Task{1, s - lag, 0, 0};
  }
  if (t < a2) return Task{1, ngroup - lag + (t - a1), 0, 0};
  return Task{2, 0, 0, 0};
}
DI int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
}  // namespace cfield

// The body of the single-launch column step, shared by the one-context
// kernel (k_column_step) and the ensemble kernel (k_column_step_ens):
// args_of(i) gives member i's arguments, claim() the next task (with its
// member), tsz the ring's slot stride in complex elements (at least the
// largest member's (Ny+2) x FS_COLS).  A task's own member fixes its sizes;
// the first tile of the next task is fetched with that task's member's.
template <int R, class ArgsOf, class Claim>
DI void column_step_body(ArgsOf args_of, Claim claim, double2* ring, int tsz) {
  using namespace cfield;
  __shared__ int s_ok;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const double2 z2 = make_double2(0.0, 0.0);
  const int j0 = lane * R;
  Task cur = claim();
  bool pre = false;   // the current task's first tile is already in flight
  int step = 0;
  // the next task's first tile (its nonlinear terms), from its own member
  auto prefetch_next = [&](double2* nslot, const Task& nxt, int n_cur, size_t ps_cur, int q0, int nvalid) {
    if (nxt.kind == 0) {
      const SolveArgs& an = args_of(nxt.mem).s;
      const int qn = nxt.g * FS_COLS;
      const FTile first = an.nl64[nxt.f] ? FTile{an.nl64[nxt.f], FT_NL, 0, 0.0}
                                         : FTile{an.nl32[nxt.f], FT_NL, 1, 0.0};
      load_ftile<R>(nslot, &first, (size_t)an.ncol, qn, min(FS_COLS, an.ncol - qn), an.n, tid);
    } else {
      load_tile<R, 16>(nslot, nullptr, ps_cur, q0, nvalid, n_cur, tid);
    }
  };
  while (cur.kind != 2) {
    const FieldArgs& A = args_of(cur.mem);
    const SolveArgs& a = A.s;
    const int n = a.n, nyp = a.nyp;
    const size_t ps = (size_t)a.ncol;          // plane stride (the Fourier pitch is 2Nkz+1)
    const double* met = A.met;
    if (cur.kind == 0) {
      const int f = cur.f;
      const int q0 = cur.g * FS_COLS;
      const int nvalid = min(FS_COLS, a.ncol - q0);
      const int q = min(q0 + w, a.ncol - 1);   // a warp past the last column works on a copy
      const int m = q / a.nk2, kq = q % a.nk2;
      const bool m00 = (q0 + w == 0);
      const double kxm = a.kx[m], kzq = a.kz[kq];
      const double k2s = kxm * kxm + kzq * kzq;
      const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
      // field kind: solve index f (0 u1, 1 u2, 2 u3, 3+n scalar n),
      // row-coefficient index (0 u1/u3, 1 u2, 2+n scalar n), explicit rows
      // [lo, hi], wall rows
      const int th = f - 3;
      const int kc_kind = f == 1 ? 1 : (f < 3 ? 0 : 2 + th);
      int lo, hi, b0, b1;
      double c0, c1;
      if (f == 0) { lo = a.jstart; hi = a.jend; b0 = a.ubc[0]; b1 = a.ubc[1]; c0 = a.uc1[0]; c1 = a.uc1[1]; }
      else if (f == 2) { lo = a.jstart; hi = a.jend; b0 = a.wbc[0]; b1 = a.wbc[1]; c0 = a.wc1[0]; c1 = a.wc1[1]; }
      else if (f == 1) { lo = 2; hi = nyp; b0 = a.vbc[0]; b1 = a.vbc[1]; c0 = a.vc1[0]; c1 = a.vc1[1]; }
      else { lo = a.jst[th]; hi = a.jet[th]; b0 = a.thbc[th][0]; b1 = a.thbc[th][1]; c0 = a.thc1[th][0]; c1 = a.thc1[th][1]; }
      const double* K = A.kc + (size_t)kc_kind * 3 * n;
      const double cfc = f >= 3 ? (a.nu / a.pr[th]) * kk : a.nu * kk;
      // mean-split correction of this field: -ikx U(j) u with U = U1 (u3,
      // scalars) or its GY interpolation I(U1) (u2); none for u1
      const double* Up = (A.mean_split && f != 0) ? A.prof + (f == 1 ? n : 0) : nullptr;
      FTile tl[FS_MAXTILES];
      const int ns = field_tiles(a, f, tl);
      if (!pre) load_ftile<R>(ring + (step & 1) * tsz, &tl[0], ps, q0, nvalid, n, tid);
      Task nxt{2, 0, 0};

      double2 cr[R], cf[R];
#pragma unroll
      for (int r = 0; r < R; ++r) { cr[r] = z2; cf[r] = z2; }
      for (int k = 0; k < ns; ++k, ++step) {
        const FTile tk = tl[k];
        double2* nslot = ring + ((step + 1) & 1) * tsz;
        if (k + 1 < ns) {
          load_ftile<R>(nslot, &tl[k + 1], ps, q0, nvalid, n, tid);
        } else {
          // claim the next task; a field task's first tile (its nonlinear
          // terms) goes in flight now, a projection's waits for its inputs
          nxt = claim();
          prefetch_next(nslot, nxt, n, ps, q0, nvalid);
        }
        wait_groups<1>();
        __syncthreads();
        double2* T = ring + (step & 1) * tsz;
        auto TV = [&](int j) -> double2 { return T[slot<R>(j, w)]; };
        switch (tk.kind) {
          case FT_OWN: {
            // cf is complete here; it leaves through this slot, overwriting the
            // field row by row: a lane takes its two neighbour rows (other
            // lanes' rows of the same column) before the warp writes anything,
            // and reads row j+1 before overwriting row j
            // (lanes whose rows lie past the system read nothing)
            const double2 h_lo = (j0 >= 1 && j0 - 1 < n) ? TV(j0 - 1) : z2;
            const double2 h_hi = j0 + R < n ? TV(j0 + R) : z2;
            __syncwarp();
            double2 um = h_lo, u = j0 < n ? TV(j0) : z2;
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              const double2 up = r == R - 1 ? h_hi : (j + 1 < n ? TV(j + 1) : z2);
              double2 c = cf[r];
              if (j >= lo && j <= hi) {
                c = c - cfc * u;
                if (Up) c = c - mul_ik(kxm * __ldg(Up + j), u);
                cr[r] = u - K[2 * n + j] * (up - u) + K[j] * (u - um);
                cr[r] = cr[r] + a.temp5 * c;
              }
              if (a.store_cf && j < n) T[slot<R>(j, w)] = c;
              um = u;
              u = up;
            }
            if (a.store_cf) {
              __syncthreads();
              store_tile<R>(T, a.cf_out[f], ps, q0, nvalid, lo, hi, tid);
            }
            break;
          }
          case FT_ADD:
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              if (j >= lo && j <= hi) cf[r] = cf[r] + tk.coef * TV(j);
            }
            break;
          case FT_BUOY:
            if (!m00) {
#pragma unroll
              for (int r = 0; r < R; ++r) {
                const int j = j0 + r;
                if (j >= lo && j <= hi)
                  cf[r] = cf[r] + tk.coef * (__ldg(met + MET_WB1 * n + j) * TV(j) +
                                             __ldg(met + MET_WB2 * n + j) * TV(j - 1));
              }
            }
            break;
          case FT_NL: {
            const float2* T32 = reinterpret_cast<const float2*>(T);
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              if (j >= lo && j <= hi) {
                double2 nl;
                if (tk.f32) { const float2 v = T32[slot<R>(j, w)]; nl = make_double2(v.x, v.y); }
                else nl = TV(j);
                cf[r] = -nl;
              }
            }
            break;
          }
          case FT_CFOLD:
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              if (j >= lo && j <= hi) cr[r] = cr[r] + a.temp3 * TV(j);
            }
            break;
          case FT_P:
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              if (j >= lo && j <= hi) {
                if (f == 0) {
                  cr[r] = cr[r] - a.temp4 * mul_ik(kxm, TV(j));
                  if (m00) cr[r].x -= a.px;
                } else if (f == 2) {
                  cr[r] = cr[r] - a.temp4 * mul_ik(kzq, TV(j));
                } else {
                  cr[r] = cr[r] - a.temp4 * __ldg(met + MET_IDY * n + j) * (TV(j) - TV(j - 1));
                }
              }
            }
            break;
          default:
            break;
        }
        __syncthreads();
      }
      // right-hand side: explicit terms on the explicit rows, wall values on
      // the wall rows (for/channel.f90:1545-1876); the matrix is in the factor
      // table
      const double v00 = m00 ? 1.0 : 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r;
        double2 d = (j >= lo && j <= hi) ? cr[r] : z2;
        if (f == 1) {
          if (b0 == 0 && (j == 1 || j == 2)) d = make_double2(c0 * v00, 0);
          if (b0 == 1 && j == 1) d = make_double2(a.dyf[1] * c0 * v00, 0);
          if (j == 0) d = z2;
          if (b1 == 0 && (j == nyp || j == nyp + 1)) d = make_double2(c1 * v00, 0);
          if (b1 == 1 && j == nyp + 1) d = make_double2(a.dyf[nyp] * c1 * v00, 0);
        } else {
          if (j == 0 || j == nyp + 1) d = z2;
          if (j == 1) d = make_double2((b0 == 0 ? c0 : a.dy[2] * c0) * v00, 0);
          if (j == nyp) d = make_double2((b1 == 0 ? c1 : a.dy[nyp] * c1) * v00, 0);
        }
        cr[r] = d;
      }
      apply_factored<R>(A.fac + (size_t)f * Fac<R>::N * 32, cr, lane);
      // The solve writes rows w0 .. Ny+1 (u2: from row 1, the others from
      // lo - 1); rows below keep their input value.
      const int w0 = f == 1 ? 1 : lo - 1;
      double2* out = ring + ((step - 1) & 1) * tsz;   // the slot of the last step
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r;
        if (j < n) out[slot<R>(j, w)] = cr[r];
      }
      __syncthreads();
      const double2* own = f < 3 ? a.cu_in[f] : a.cth_in[th];
      store_tile<R>(out, f < 3 ? a.cu_out[f] : a.cth_out[th], ps, q0, nvalid, 0, n - 1, tid, own, w0);
      // publish a velocity field's completion to its group's projection: every
      // thread's stores are ordered before the count (the next task's second
      // tile also goes to this slot only after the barrier)
      __threadfence();
      __syncthreads();
      if (f < 3 && tid == 0) atomicAdd(A.sched + SCHED_DONE + cur.g, 1);
      pre = nxt.kind == 0;
      cur = nxt;
    } else {
      double2* const* cu = a.cu_out;
      const void* src[7] = {cu[0], cu[2], cu[1], cu[0], cu[2], cu[1], a.cp_in};
      const double ih = 1.0 / a.temp4;
      const int g = cur.g;
      const int q0 = g * FS_COLS;
      const int nvalid = min(FS_COLS, a.ncol - q0);
      const int q = min(q0 + w, a.ncol - 1);
      const int m = q / a.nk2, kq = q % a.nk2;
      const bool m00 = (q0 + w == 0);
      const double kxm = a.kx[m], kzq = a.kz[kq];
      // wait (bounded) until the three velocity solves of this group are done
      if (tid == 0) {
        int ok = 1;
        long long it = 0;
        while (ld_acquire(A.sched + SCHED_DONE + g) < A.need) {
          if (*(volatile int*)(A.sched + SCHED_STATUS) != 0 || ++it > A.max_spins) {
            ok = 0;
            atomicExch(A.sched + SCHED_STATUS, 1);
            break;
          }
          __nanosleep(100);
        }
        __threadfence();
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) {   // timed out: this group is left as it is
        cur = claim();
        pre = false;
        continue;
      }
      load_tile<R, 16>(ring + (step & 1) * tsz, src[0], ps, q0, nvalid, n, tid);
      Task nxt{2, 0, 0};
      double2 d[R];
#pragma unroll
      for (int r = 0; r < R; ++r) d[r] = z2;
      double2 phm = z2;
      for (int k = 0; k < 7; ++k, ++step) {
        double2* nslot = ring + ((step + 1) & 1) * tsz;
        if (k + 1 < 7) load_tile<R, 16>(nslot, src[k + 1], ps, q0, nvalid, n, tid);
        else {
          nxt = claim();
          prefetch_next(nslot, nxt, n, ps, q0, nvalid);
        }
        wait_groups<1>();
        __syncthreads();
        double2* T = ring + (step & 1) * tsz;
        if (k < 3) {
          // divergence ik.u1 + ik.u3 + (u2(j+1) - u2(j))/dyf(j), rows 1..Ny,
          // in the order the solves of the fused step accumulated it
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= 1 && j <= nyp) {
              if (k == 0) d[r] = d[r] + mul_ik(kxm, T[slot<R>(j, w)]);
              else if (k == 1) d[r] = d[r] + mul_ik(kzq, T[slot<R>(j, w)]);
              else d[r] = d[r] + __ldg(met + MET_IDYF * n + j) * (T[slot<R>(j + 1, w)] - T[slot<R>(j, w)]);
            }
          }
          if (k == 2) {
            // Poisson rows: interior 1/(dy dyf) terms, Neumann walls, phi(1) = 0
            // for the (0,0) mode
            double al[R], cm[R];
            const double k2n = -kxm * kxm - kzq * kzq;
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int j = j0 + r;
              double am = 0.0, cc = 0.0;
              if (j >= 1 && j <= nyp) { am = __ldg(met + MET_PA * n + j); cc = __ldg(met + MET_PC * n + j); }
              if (j == 1) { am = 0; cc = m00 ? 0.0 : -1.0; d[r] = z2; }
              if (j == nyp) { am = 1; cc = 0; d[r] = z2; }
              al[r] = am;
              cm[r] = cc;
            }
            csolve2::warp_tridiag_b<R>([&](int r) -> double& { return al[r]; }, [&](int r) -> double {
              const int j = j0 + r;
              return (j == 1) ? 1.0 : (j == nyp ? -1.0 : ((j > 1 && j < nyp) ? k2n + __ldg(met + MET_PB0 * n + j) : 1.0));
            }, [&](int r) -> double& { return cm[r]; }, d, lane);
            phm = shfl_up2(d[R - 1], 1);   // phi of the row below the lane's first
          }
        } else if (k < 6) {
          const int comp = k == 3 ? 0 : (k == 4 ? 2 : 1);
          if (a.keep[0]) {
            store_tile<R>(T, a.keep[comp], ps, q0, nvalid, 1, nyp, tid);
            __syncthreads();
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (comp != 1 && j >= 1 && j <= nyp) {
              double2& u = T[slot<R>(j, w)];
              u = u - mul_ik(comp == 0 ? kxm : kzq, d[r]);
            }
            if (comp == 1 && j >= 2 && j <= nyp) {
              double2& u = T[slot<R>(j, w)];
              u = u - __ldg(met + MET_IDY * n + j) * (d[r] - (r == 0 ? phm : d[r - 1]));
            }
          }
          __syncthreads();
          store_tile<R>(T, cu[comp], ps, q0, nvalid, comp == 1 ? 2 : 1, nyp, tid);
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= a.jstart && j <= a.jend) {
              double2& p = T[slot<R>(j, w)];
              p = p + ih * d[r];
            }
          }
          __syncthreads();
          store_tile<R>(T, a.cp_out, ps, q0, nvalid, 0, n - 1, tid);
        }
        __syncthreads();
      }
      pre = nxt.kind == 0;
      cur = nxt;
    }
  }
  wait_groups<0>();
}

template <int R>
__global__ void __launch_bounds__(FS_THREADS, fs_min_blocks<R>()) k_column_step(const __grid_constant__ FieldArgs A) {
  using namespace cfield;
  extern __shared__ __align__(16) unsigned char fs_smem[];
  __shared__ int s_next;
  const int ngroup = (A.s.ncol + FS_COLS - 1) / FS_COLS;
  const int lag = min(A.lag, ngroup);
  auto args_of = [&](int) -> const FieldArgs& { return A; };
  auto claim = [&]() -> Task {
    if (threadIdx.x == 0) s_next = atomicAdd(A.sched + SCHED_COUNTER, 1);
    __syncthreads();
    return decode_task(s_next, ngroup, A.nf, lag);
  };
  column_step_body<R>(args_of, claim, reinterpret_cast<double2*>(fs_smem), A.s.n * FS_COLS);
}

// ---- k_column_step_ens -------------------------------------------------------------
// The column step of every member of an ensemble whose systems have R rows
// per lane, in one persistent launch: a member table, and one task counter
// over all members' tasks (member i's tasks are numbers prefix[i] ..
// prefix[i+1]-1, in k_column_step's order).  Each member keeps its own
// scheduler words (per-group counts, status) and wait bound; a projection
// task waits, bounded, on its own member's group counts only, for tasks
// claimed before it by running blocks, so the wait ends as in k_column_step.
struct EnsColArgs {
  const FieldArgs* mem;   // [nmem] member arguments (device)
  const int* prefix;      // [nmem + 1] first task of each member (device)
  int* counter;           // the launch's task counter (zeroed before it)
  int nmem;
  int tsz;                // ring slot stride: 32 R FS_COLS
};

template <int R>
__global__ void __launch_bounds__(FS_THREADS, fs_min_blocks<R>()) k_column_step_ens(const __grid_constant__ EnsColArgs E) {
  using namespace cfield;
  extern __shared__ __align__(16) unsigned char fs_smem[];
  __shared__ int s_next, s_mem;
  auto args_of = [&](int i) -> const FieldArgs& { return E.mem[i]; };
  auto claim = [&]() -> Task {
    if (threadIdx.x == 0) {
      const int t = atomicAdd(E.counter, 1);
      int lo = 0, hi = E.nmem;   // the member i with prefix[i] <= t < prefix[i+1]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (E.prefix[mid] <= t) lo = mid; else hi = mid;
      }
      s_next = t;
      s_mem = t < E.prefix[E.nmem] ? lo : -1;
    }
    __syncthreads();
    const int i = s_mem;
    if (i < 0) return Task{2, 0, 0, 0};
    const FieldArgs& A = E.mem[i];
    const int ngroup = (A.s.ncol + FS_COLS - 1) / FS_COLS;
    Task k = decode_task(s_next - E.prefix[i], ngroup, A.nf, min(A.lag, ngroup));
    k.mem = i;
    return k;
  };
  column_step_body<R>(args_of, claim, reinterpret_cast<double2*>(fs_smem), E.tsz);
}
