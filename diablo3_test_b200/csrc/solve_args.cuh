// Argument blocks of the column kernels (k_column_tiles, k_column_solve,
// k_rem_div, k_factor), shared by the kernels and the host code that fills
// them.
#pragma once
#include "common.cuh"

#define SOLVE_MAXTH 8
#define SOLVE_NF (3 + SOLVE_MAXTH)

struct SolveArgs {
  int nyp, n;               // Nyp, Ny+2
  int nkx1, nk2, kp, ncol;  // stored x modes, packed z modes, pitch, columns
  int nth, rk;
  double temp1, temp2, temp3, temp4, temp5;
  double nu, beta, nu_v, roinvd;  // nu, horizontal Laplacian exponent, nu_v_scale, Ro_inv/delta
  double grav_x, grav_y, grav_z;
  double px;                // subtracted from cr1 at (0,0): temp4*(px0 [+ oscillation])
  int jstart, jend;
  int ubc[2], vbc[2], wbc[2];
  double uc1[2], vc1[2], wc1[2];  // wc1[1] is the (possibly transient) top value
  int front;                // thermal-wind advection (flavor 'Front')
  double ly, front_coef;    // Ly, delta/Ro_inv
  int jst[SOLVE_MAXTH], jet[SOLVE_MAXTH];
  int thbc[SOLVE_MAXTH][2];
  double thc1[SOLVE_MAXTH][2];
  double pr[SOLVE_MAXTH], dthdx[SOLVE_MAXTH], dthdz[SOLVE_MAXTH];
  const double* dy;
  const double* dyf;
  const double* gy;
  const double* gyf;
  const double* kx;
  const double* kz;
  const double2* cu_in[3];
  const double2* cth_in[SOLVE_MAXTH];
  const double2* cp_in;
  const double2* cf_in[SOLVE_NF];
  double2* cu_out[3];
  double2* cth_out[SOLVE_MAXTH];
  double2* cp_out;
  double2* cf_out[SOLVE_NF];
  const double2* nl64[SOLVE_NF];
  const float2* nl32[SOLVE_NF];
  int store_cf;             // 0 on the last substep (cf is not read again)
  double2* keep[3];         // if set: the solved u1, u2, u3 before the projection (courant)
};

#define T2_COLS 4
#define T2_PITCH 4      // complex elements per tile row (unpadded; see tix)
#define T2_MAXSTEPS 96

enum TileOp {
  OP_OWN_U13 = 1,  // u1/u3 own field: cf = -nu kk u ; cr = u + t1v*lap(u)      arg: comp
  OP_OWN_U2,       // u2 own field (staggered metric)
  OP_OWN_TH,       // scalar own field                                        arg: scalar
  OP_ADD_CF,       // cf += coef * tile
  OP_BUOY,         // cf += grav_y * interp_y(tile), rows 2..Nyp, not the (0,0) mode
  OP_NL,           // cf -= tile ; store cf ; cr += temp5*cf                  arg: fp32 flag
  OP_CFOLD,        // cr += temp3 * tile
  OP_SOLVE,        // pressure gradient, matrix + wall rows, solve, store     arg: field kind
  OP_POISSON,      // phi from the accumulated divergence
  OP_PROJ,         // tile = new velocity; subtract grad phi; store; src2: keep the tile  arg: comp
  OP_CP            // cp_out = cp_in + phi/temp4
};

struct TileStep {
  int op, arg;
  double coef;
  const void* src;   // tile source (nullptr: no tile)
  void* dst;         // store target (cf_out, cu_out, ...)
  const void* src2;  // rows outside the write range are copied from here (OP_SOLVE)
};

// Row coefficients precomputed on the host (the reference's expressions,
// for/channel.f90:664-670, :726-733, :782-788, :969-976):
//   kc[kind][3][n]  implicit rows A, B, C of this substep; kind 0 = u1/u3,
//                   1 = u2, 2+n = scalar n.  The explicit Crank-Nicolson half is
//                   u - C (u(j+1) - u(j)) + A (u(j) - u(j-1)).
//   met[7][n]       Poisson A, C, B without k^2; 1/dy; 1/dyf; buoyancy weights
//                   dyf(j-1)/(2dy(j)), dyf(j)/(2dy(j)).
enum { MET_PA = 0, MET_PC, MET_PB0, MET_IDY, MET_IDYF, MET_WB1, MET_WB2, MET_N };

struct Solve2Args {
  SolveArgs s;
  const double* kc;
  const double* met;
  const double* fac;   // factored u1, u2, u3, scalar systems of this substep (see k_factor)
  // 1: the nonlinear tiles (FP32) of the u2, u3 and scalar equations were
  // computed with u1 minus its mean profile U1(y) (the (0,0) mode); the
  // products with U1 are linear in the state and are added here in FP64:
  //   u3: ikx U1 u3,   u2: ikx I(U1) u2,   scalar: ikx U1 th
  // with I the GYF-to-GY interpolation of for/channel.f90:356-375.  (The u1
  // equation's FP64 NL carries its own mean terms, see ZFwdArgs.)
  int mean_split;
  const double* prof;  // [2][n]: U1(j), I(U1)(j) (written by the z-forward epilogue)
  int nstep;
  TileStep steps[T2_MAXSTEPS];
};

// Columns (one warp each) per block of the field-split column step
// (kernels_field.cuh); the host sizes the step's scheduler by it.
#define FS_COLS 8
#define FS_THREADS (32 * FS_COLS)
