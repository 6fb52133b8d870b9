// thickness.cu -- the consumers of the velocities inside a time step, on the device:
// the explicit ice-thickness update (calc_dHi_dt, ice_thickness_module.f90:26-300,
// with apply_ice_thickness_BC :728-931), the floating margin fraction
// (general_ice_model_data_module.f90:784-865), the advective time-step limit and the
// predictor/corrector stages of run_ice_dynamics_pc (ice_dynamics_module.f90:243-432,
// 726-816).  The time-step control (dt_crit, pc_zeta, pc_eta, the event clock) stays
// host logic around these calls.
//
// Compiled without FMA contraction: every value is the reference's sequence of
// IEEE operations, bit for bit.  The outflux limitation of the reference runs in
// place in loop order, but a face is rescaled only by its upwind cell and a cell's
// factor depends only on its own outfluxes, so one launch per stage reproduces it.
#include <cmath>
#include <cstdio>
#include "ctx.hpp"

namespace diva {
namespace {

#define IDX2D                                                            \
  const int j = blockIdx.x * blockDim.x + threadIdx.x;                   \
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
#define G2T grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream

// surface_elevation and Hi_from_Hb_and_Hs (utilities_module.f90:138-183)
__device__ __forceinline__ double surface_elev(double Hi, double Hb, double SL) {
  return Hi + max_ref(SL - kRhoI / kRhoSW * Hi, Hb);
}
__device__ __forceinline__ double hi_from_hb_hs(double Hb, double Hs, double SL) {
  const double Hs_float = Hb + (SL - Hb) * kRhoSW / kRhoI;
  if (Hs > Hs_float) return Hs - Hb;
  return (Hs - SL) / (1.0 - kRhoI / kRhoSW);
}

__global__ void k_float_margin(Dims d, const double* Hi, const int* ice, const int* cf, const int* shelf,
                               double* fmf, double* Heff) {
  IDX2D
  if (j < 1 || j > d.ny - 2 || i >= d.nx) return;
  const long long q = d.at(j, i);
  fmf[q] = ice[q] == 1 ? 1.0 : 0.0;
  Heff[q] = ice[q] == 1 ? Hi[q] : 0.0;
  if (!(cf[q] == 1 && shelf[q] == 1)) return;
  bool inner = false;
  double Hmax = 0.0;
  for (int ii = (i > 0 ? i - 1 : 0); ii <= (i < d.nx - 1 ? i + 1 : d.nx - 1); ++ii)
    for (int jj = j - 1; jj <= j + 1; ++jj) {
      const long long p = d.at(jj, ii);
      if (ice[p] == 1 && cf[p] == 0) {
        inner = true;
        Hmax = max_ref(Hmax, Hi[p]);
      }
    }
  if (!inner || Hmax < Hi[q]) {
    fmf[q] = 1.0;
    Heff[q] = Hi[q];
    return;
  }
  fmf[q] = Hi[q] / Hmax;
  Heff[q] = Hmax;
}

// upwind fluxes (:91-120), volumes of ice moved during dt
__global__ void k_fluxes(Dims d, double dt, const double* u, const double* v, const double* Hi, double* Qx,
                         double* Qy) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (i < d.nx - 1) {
    const double uu = u[q];
    Qx[q] = uu * (uu > 0.0 ? Hi[q] : Hi[d.at(j, i + 1)]) * d.dx * dt;
  }
  if (j < d.ny - 1) {
    const double vv = v[q];
    Qy[q] = vv * (vv > 0.0 ? Hi[q] : Hi[d.at(j + 1, i)]) * d.dx * dt;
  }
}

// mass balance volume and the outflux rescale factor of each cell (:175-245)
__global__ void k_cell_budget(Dims d, double dt, const double* Hi, const double* smb, const double* bmb,
                              const double* fmf, const int* cf, const int* shelf, const int* ocean, const double* Qx,
                              const double* Qy, double* mb, double* rf) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double dx = d.dx;
  double m;
  if (cf[q] == 1 && shelf[q] == 1) m = (smb[q] + bmb[q]) * dx * dx * dt * fmf[q];
  else if (ocean[q] == 1 && shelf[q] == 0) m = 0.0;
  else m = (smb[q] + bmb[q]) * dx * dx * dt;
  const double avail = Hi[q] * dx * dx;
  double out = 0.0;
  if (i > 0 && !(Qx[d.at(j, i - 1)] > 0.0)) out = out - Qx[d.at(j, i - 1)];
  if (i < d.nx - 1 && !(Qx[q] < 0.0)) out = out + Qx[q];
  if (j > 0 && !(Qy[d.at(j - 1, i)] > 0.0)) out = out - Qy[d.at(j - 1, i)];
  if (j < d.ny - 1 && !(Qy[q] < 0.0)) out = out + Qy[q];
  double r = 1.0;
  if (-m >= avail) {
    m = -avail;
    r = 0.0;
  }
  if (out > avail + m) r = (avail + m) / out;
  mb[q] = m;
  rf[q] = r;
}

// each face rescaled by its upwind cell (:246-262)
__global__ void k_rescale_faces(Dims d, const double* rf, double* Qx, double* Qy) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (i < d.nx - 1) {
    const double Q = Qx[q];
    if (Q > 0.0 && rf[q] < 1.0) Qx[q] = Q * rf[q];
    else if (Q < 0.0 && rf[d.at(j, i + 1)] < 1.0) Qx[q] = Q * rf[d.at(j, i + 1)];
  }
  if (j < d.ny - 1) {
    const double Q = Qy[q];
    if (Q > 0.0 && rf[q] < 1.0) Qy[q] = Q * rf[q];
    else if (Q < 0.0 && rf[d.at(j + 1, i)] < 1.0) Qy[q] = Q * rf[d.at(j + 1, i)];
  }
}

// rate of change and thickness at t + dt (:266-290)
__global__ void k_dhdt(Dims d, double dt, const double* Hi, const double* mb, const double* Qx, const double* Qy,
                       double* dH, double* Hn) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double dx = d.dx;
  double r = mb[q] / (dx * dx * dt);
  if (i > 0) r = r + Qx[d.at(j, i - 1)] / (dx * dx * dt);
  if (i < d.nx - 1) r = r - Qx[q] / (dx * dx * dt);
  if (j > 0) r = r + Qy[d.at(j - 1, i)] / (dx * dx * dt);
  if (j < d.ny - 1) r = r - Qy[q] / (dx * dx * dt);
  r = max_ref(r, -Hi[q] / dt);
  dH[q] = r;
  Hn[q] = Hi[q] + r * dt;
}

// apply_ice_thickness_BC (:728-931), one block: the sides in the reference's order,
// west, east, south, north, so corners and 'infinite' neighbours see the earlier sides
struct HBC {
  int side[4];
  int diva;
};
__global__ void k_thickness_bc(Dims d, HBC b, double dt, const double* Hi, const double* Hb, const double* SL,
                               double* Hn, double* dH) {
  for (int s = 0; s < 4; ++s) {
    const bool xs = s < 2;
    const int n = xs ? d.ny : d.nx;
    const int edge = s == 0 ? 0 : s == 1 ? d.nx - 1 : s == 2 ? 0 : d.ny - 1;
    const int inner = s == 0 ? 1 : s == 1 ? d.nx - 2 : s == 2 ? 1 : d.ny - 2;
    const int opp = s == 0 ? d.nx - 2 : s == 1 ? 1 : s == 2 ? d.ny - 2 : 1;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const long long q = xs ? d.at(k, edge) : d.at(edge, k);
      const long long qi = xs ? d.at(k, inner) : d.at(inner, k);
      const long long qo = xs ? d.at(k, opp) : d.at(opp, k);
      switch (b.side[s]) {
        case DIVA_HBC_ZERO:
          Hn[q] = 0.0;
          dH[q] = -Hi[q] / dt;
          if (b.diva) {
            Hn[qi] = 0.0;
            dH[qi] = -Hi[qi] / dt;
          }
          break;
        case DIVA_HBC_INFINITE: {
          const double Hs_nb = surface_elev(Hn[qi], Hb[qi], SL[qi]);
          Hn[q] = hi_from_hb_hs(Hb[q], Hs_nb, SL[q]);
          dH[q] = (Hn[q] - Hi[q]) / dt;
          break;
        }
        case DIVA_HBC_PERIODIC:
          Hn[q] = Hi[qo];
          dH[q] = (Hn[q] - Hi[q]) / dt;
          break;
        case DIVA_HBC_FIXED:
          Hn[q] = Hi[q];
          dH[q] = 0.0;
          break;
        default:
          break;
      }
    }
    __syncthreads();
  }
}

// min (sign < 0) or max (sign > 0) over blocks: per-block partials, then one block
__device__ __forceinline__ double pick(double a, double b, int sign) { return sign < 0 ? min_ref(a, b) : max_ref(a, b); }
__device__ void block_extreme(double v, int sign, double* out) {
  __shared__ double sh[256];
  const int t = threadIdx.x + threadIdx.y * blockDim.x, n = blockDim.x * blockDim.y;
  sh[t] = v;
  __syncthreads();
  for (int s = n / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] = pick(sh[t], sh[t + s], sign);
    __syncthreads();
  }
  if (t == 0) *out = sh[0];
}

// calc_critical_timestep_adv (ice_dynamics_module.f90:726-762), per block
__global__ void k_crit_adv(Dims d, double init, const double* u, const double* v, double* part) {
  IDX2D
  double m = init;
  if (j >= 1 && j <= d.ny - 2 && i >= 1 && i <= d.nx - 2) {
    const long long q = d.at(j, i);
    m = min_ref(m, d.dx / (fabs(u[q]) + fabs(v[q])));
  }
  block_extreme(m, -1, &part[blockIdx.y * gridDim.x + blockIdx.x]);
}
// calc_critical_timestep_SIA (ice_dynamics_module.f90:651-725): the diffusive limit
// dx^2 / (6 D_SIA) from the depth-averaged SIA velocities of sheet faces, and the 3D
// advective limit dx / (|u| + |v|) of every layer, per-block minima
struct SiaDt {
  Dims d;
  Zeta zt;
  double init;
  const int* sheet;
  const double *us, *vs, *Hcx, *Hcy, *sx, *sy, *u3, *v3;
};
__device__ __forceinline__ double vavg_layers(const Zeta& zt, const double* f, long long stride) {
  double s = 0.0;   // vertical_average, utilities_module.f90:97-123
  for (int k = 0; k < zt.nz - 1; ++k) s = s + 0.5 * (f[(k + 1) * stride] + f[k * stride]) * (zt.z[k + 1] - zt.z[k]);
  return s;
}
__global__ void k_crit_sia(SiaDt a, double* part) {
  IDX2D
  const Dims& d = a.d;
  double m = a.init;
  if (j < d.ny && i < d.nx) {
    const long long q = d.at(j, i), P = d.plane;
    double D = 1E-9;
    if (i < d.nx - 1 && a.sheet[q] == 1 && a.sheet[d.at(j, i + 1)] == 1)
      D = max_ref(D, fabs(vavg_layers(a.zt, a.us + q, P) * a.Hcx[q] / a.sx[q]));
    if (j < d.ny - 1 && a.sheet[q] == 1 && a.sheet[d.at(j + 1, i)] == 1)
      D = max_ref(D, fabs(vavg_layers(a.zt, a.vs + q, P) * a.Hcy[q] / a.sy[q]));
    m = min_ref(m, d.dx * d.dx / (6.0 * D));
    for (int k = 0; k < d.nz; ++k) {
      const double* u = a.u3 + k * P;
      const double* v = a.v3 + k * P;
      const double ua = i == 0 ? fabs(u[d.at(j, 0)]) : i == d.nx - 1 ? fabs(u[d.at(j, d.nx - 2)])
                                                                     : max_ref(fabs(u[d.at(j, i - 1)]), fabs(u[q]));
      const double va = j == 0 ? fabs(v[d.at(0, i)]) : j == d.ny - 1 ? fabs(v[d.at(d.ny - 2, i)])
                                                                     : max_ref(fabs(v[d.at(j - 1, i)]), fabs(v[q]));
      m = min_ref(m, d.dx / (ua + va));
    }
  }
  block_extreme(m, -1, &part[blockIdx.y * gridDim.x + blockIdx.x]);
}

__global__ void k_extreme_final(const double* part, int nb, double init, int sign, double* out) {
  double m = init;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) m = pick(m, part[b], sign);
  block_extreme(m, sign, out);
}

__global__ void k_pc_predict(Dims d, double dt, double zeta, double* Hi, const double* hn, const double* hm,
                             double* pred, double* old) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  pred[q] = max_ref(0.0, Hi[q] + dt * ((1.0 + zeta / 2.0) * hn[q] - (zeta / 2.0) * hm[q]));
  old[q] = Hi[q];
  Hi[q] = pred[q];
}

__global__ void k_pc_correct(Dims d, double dt, const double* Hi, const double* old, const double* hn,
                             const double* hs, double* corr, double* dH) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  corr[q] = max_ref(0.0, old[q] + 0.5 * dt * (hn[q] + hs[q]));
  dH[q] = (corr[q] - Hi[q]) / dt;
}

// calc_pc_truncation_error (:763-816), per block
__global__ void k_pc_tau(Dims d, double dt, double zeta, double eta_min, const double* corr, const double* pred,
                         const int* sheet, const int* gl, double* tau, double* part) {
  IDX2D
  double e = eta_min;
  if (j >= 1 && j <= d.ny - 2 && i >= 1 && i <= d.nx - 2) {
    const long long q = d.at(j, i);
    const double t = fabs(zeta * (corr[q] - pred[q]) / ((3.0 * zeta + 3.0) * dt));
    tau[q] = t;
    bool near_gl = false;
    for (int ii = i - 1; ii <= i + 1; ++ii)
      for (int jj = j - 1; jj <= j + 1; ++jj) near_gl = near_gl || gl[d.at(jj, ii)] != 0;
    if (sheet[q] == 1 && !near_gl) e = max_ref(e, t);
  }
  block_extreme(e, 1, &part[blockIdx.y * gridDim.x + blockIdx.x]);
}

// Hi_tplusdt_a, the fixed-geometry options of update_ice_thickness (:449-540: a cell keeps
// its thickness when it is shelf / sheet / grounding line by the 3 x 3 mask test), then
// Hi_a = max(0, Hi_tplusdt_a)
struct FixFlags {
  int shelf, sheet, gl;
};
__global__ void k_pc_finish(Dims d, double dt, double* Hi, const double* dH, double* Hn, FixFlags fx,
                            const int* shelf, const int* sheet) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  double hn = max_ref(0.0, Hi[q] + dt * dH[q]);
  if (fx.shelf | fx.sheet | fx.gl) {
    bool nb_shelf = false, nb_sheet = false;
    for (int ii = (i > 0 ? i - 1 : 0); ii <= (i < d.nx - 1 ? i + 1 : d.nx - 1); ++ii)
      for (int jj = (j > 0 ? j - 1 : 0); jj <= (j < d.ny - 1 ? j + 1 : d.ny - 1); ++jj) {
        nb_shelf = nb_shelf || shelf[d.at(jj, ii)] == 1;
        nb_sheet = nb_sheet || sheet[d.at(jj, ii)] == 1;
      }
    const bool sh = shelf[q] == 1, sg = sheet[q] == 1;
    if (fx.shelf && (sh || (sg && nb_shelf))) hn = Hi[q];
    if (fx.sheet && (sg || (sh && nb_sheet))) hn = Hi[q];
    if (fx.gl && ((sg && nb_shelf) || (sh && nb_sheet))) hn = Hi[q];
  }
  Hn[q] = hn;
  Hi[q] = max_ref(0.0, hn);
}

// ---- remove_unconnected_shelves (:932-1044) -----------------------------------------
// The reference searches depth-first from the interior shelf cells next to sheet ice
// through 4-connected shelf cells; the reached set is that connected component, which
// label propagation gives the same: seeds, then repeated spreading (iterated inside a
// block over its tile, relaunched until nothing changes), then the removal.
constexpr int kSX = 32, kSY = 8;
__global__ void k_shelf_seed(Dims d, const int* shelf, const int* sheet, int* reach) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  int r = 0;
  if (j >= 1 && j <= d.ny - 2 && i >= 1 && i <= d.nx - 2 && shelf[q] == 1)
    r = (sheet[d.at(j, i + 1)] == 1 || sheet[d.at(j, i - 1)] == 1 || sheet[d.at(j + 1, i)] == 1 ||
         sheet[d.at(j - 1, i)] == 1) ? 1 : 0;
  reach[q] = r;
}
__global__ void k_shelf_spread(Dims d, const int* shelf, int* reach, int* changed) {
  __shared__ int sr[kSY + 2][kSX + 2];
  __shared__ int ss[kSY + 2][kSX + 2];
  const int j0 = blockIdx.x * kSX, i0 = blockIdx.y * kSY;
  for (int t = threadIdx.y * kSX + threadIdx.x; t < (kSX + 2) * (kSY + 2); t += kSX * kSY) {
    const int lj = t % (kSX + 2), li = t / (kSX + 2);
    const int j = j0 + lj - 1, i = i0 + li - 1;
    const bool in = j >= 0 && j < d.ny && i >= 0 && i < d.nx;
    // a reached cell spreads only if it is shelf itself
    sr[li][lj] = in ? (reach[d.at(j, i)] && shelf[d.at(j, i)] == 1) : 0;
    ss[li][lj] = in ? (shelf[d.at(j, i)] == 1) : 0;
  }
  __syncthreads();
  const int lj = threadIdx.x + 1, li = threadIdx.y + 1;
  const int j = j0 + threadIdx.x, i = i0 + threadIdx.y;
  const bool mine = j < d.ny && i < d.nx;
  int any = 0;
  for (int it = 0; it < kSX * kSY + 4; ++it) {
    int ch = 0;
    if (mine && ss[li][lj] && !sr[li][lj] && (sr[li - 1][lj] | sr[li + 1][lj] | sr[li][lj - 1] | sr[li][lj + 1])) ch = 1;
    __syncthreads();
    if (ch) sr[li][lj] = 1;
    any |= ch;
    if (!__syncthreads_or(ch)) break;
  }
  if (mine && any) {
    reach[d.at(j, i)] = 1;
    atomicOr(changed, 1);
  }
}
// then the no-ice mask (:586-592) and, with do_remove_shelves, all floating ice (:600-608)
// apply_prescribed_retreat_mask (calving_module.f90:125-136): the mask at the model time
__global__ void k_retreat_interp(Dims d, double wt0, const double* m0, const double* m1, double* m) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  m[q] = (wt0 * m0[q]) + ((1.0 - wt0) * m1[q]);
}

// (:139-164): cap the thickness where the mask has retreat, and at interior cells next to it
__global__ void k_retreat_apply(Dims d, const double* m, const double* Href, double* Hi) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  bool cap = m[q] < 0.999;
  if (!cap && i > 0 && i < d.nx - 1 && j > 0 && j < d.ny - 1)
    for (int di = -1; di <= 1; ++di)
      for (int dj = -1; dj <= 1; ++dj)
        if ((di || dj) && m[d.at(j + dj, i + di)] < 0.999) cap = true;
  if (cap) Hi[q] = fmin(Hi[q], Href[q] * m[q]);
}

// threshold_thickness_calving (calving_module.f90:62-91): calving-front cells whose
// effective thickness is below the threshold lose their ice
__global__ void k_calve_threshold(Dims d, const int* cf, const double* Heff, double thr, double* Hi) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (cf[q] == 1 && Heff[q] < thr) Hi[q] = 0.0;
}

// the removal options of update_ice_thickness with reference geometries (:613-635)
struct RefGeo {
  int larger_than_pd, shelf_edge;
  double shelf_min_height;
  const double *Hi_pd, *Hb_pd, *Hi_eq, *Hb_eq;
};

__global__ void k_shelf_remove(Dims d, const int* shelf, const int* reach, const int* noice, int remove_floating,
                               const double* Hb, const double* SL, RefGeo rg, double* Hi) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (shelf[q] == 1 && !reach[q]) Hi[q] = 0.0;
  if (noice[q] == 1) Hi[q] = 0.0;
  if (remove_floating && Hi[q] < (SL[q] - Hb[q]) * kRhoSW / kRhoI) Hi[q] = 0.0;
  if (rg.larger_than_pd && rg.Hi_pd[q] == 0.0 && rg.Hb_pd[q] < 0.0) Hi[q] = 0.0;
  if (rg.shelf_edge && rg.Hi_eq[q] == 0.0 && rg.Hb_eq[q] < rg.shelf_min_height) Hi[q] = 0.0;
}

// ---- the semi-implicit scheme (calc_dHi_dt_semiimplicit, :302-727) ---------------------
// Per cell a row of the implicit system: identity (mass-balance-only or explicit cells)
// or the over-implicit upwind row (fs = 2.5).  The matrix is column diagonally dominant
// (the 1/dt term), and is solved by BiCGStab with a Jacobi preconditioner.
struct HSI {
  double *d, *cw, *ce, *cs, *cn, *b, *x;
};
__global__ void k_hsi_rows(Dims dm, double dt, const double* Hi, const double* u, const double* v, const double* smb,
                           const double* bmb, const double* fmf, const int* ice, const int* shelf, const int* ocean,
                           const int* cf, HSI h) {
  IDX2D
  if (j >= dm.ny || i >= dm.nx) return;
  const int nx = dm.nx, ny = dm.ny;
  const double fs = 2.5, dx = dm.dx;
  const int im1 = i > 0 ? i - 1 : 0, ip1 = i < nx - 1 ? i + 1 : nx - 1;
  const int jm1 = j > 0 ? j - 1 : 0, jp1 = j < ny - 1 ? j + 1 : ny - 1;
  const long long q = dm.at(j, i), qw = dm.at(j, im1), qe = dm.at(j, ip1), qs = dm.at(jm1, i), qn = dm.at(jp1, i);
  int scheme;
  if (ice[q] == 0 && ice[qw] == 0 && ice[qe] == 0 && ice[qs] == 0 && ice[qn] == 0) scheme = 0;
  else if (shelf[q] == 1 && ((ocean[qw] == 1 && ice[qw] == 0) || (ocean[qe] == 1 && ice[qe] == 0) ||
                             (ocean[qs] == 1 && ice[qs] == 0) || (ocean[qn] == 1 && ice[qn] == 0))) scheme = 1;
  else if (ocean[q] == 1 && ice[q] == 0 && (shelf[qw] == 1 || shelf[qe] == 1 || shelf[qs] == 1 || shelf[qn] == 1))
    scheme = 1;
  else scheme = 2;
  double mb;
  if (cf[q] == 1 && shelf[q] == 1) mb = (smb[q] + bmb[q]) * fmf[q];
  else if (ocean[q] == 1 && shelf[q] == 0) mb = 0.0;
  else mb = smb[q] + bmb[q];
  bool cut_w = false, cut_e = false, cut_s = false, cut_n = false;
  if (i > 0) {
    if (shelf[q] == 1 && ocean[qw] == 1 && ice[qw] == 0) cut_w = fmf[q] < 1.0;
    else if (shelf[qw] == 1 && ocean[q] == 1 && ice[q] == 0) cut_w = fmf[qw] < 1.0;
  }
  if (i < nx - 1) {
    if (shelf[q] == 1 && ocean[qe] == 1 && ice[qe] == 0) cut_e = fmf[q] < 1.0;
    else if (shelf[qe] == 1 && ocean[q] == 1 && ice[q] == 0) cut_e = fmf[qe] < 1.0;
  }
  if (j > 0) {
    if (shelf[q] == 1 && ocean[qs] == 1 && ice[qs] == 0) cut_s = fmf[q] < 1.0;
    else if (shelf[qs] == 1 && ocean[q] == 1 && ice[q] == 0) cut_s = fmf[qs] < 1.0;
  }
  if (j < ny - 1) {
    if (shelf[q] == 1 && ocean[qn] == 1 && ice[qn] == 0) cut_n = fmf[q] < 1.0;
    else if (shelf[qn] == 1 && ocean[q] == 1 && ice[q] == 0) cut_n = fmf[qn] < 1.0;
  }
  double d = 1.0, cw = 0.0, ce = 0.0, cs = 0.0, cn = 0.0, b, x0;
  if (scheme == 0) {
    b = max_ref(0.0, Hi[q] + (mb * dt));
    x0 = b;
  } else if (scheme == 1) {
    double Qw = 0.0, Qe = 0.0, Qs = 0.0, Qn = 0.0;
    if (i > 0) { const double uu = u[dm.at(j, i - 1)]; Qw = uu * (uu > 0.0 ? Hi[qw] : Hi[q]) / dx; }
    if (i < nx - 1) { const double uu = u[q]; Qe = -uu * (uu > 0.0 ? Hi[q] : Hi[qe]) / dx; }
    if (j > 0) { const double vv = v[dm.at(j - 1, i)]; Qs = vv * (vv > 0.0 ? Hi[qs] : Hi[q]) / dx; }
    if (j < ny - 1) { const double vv = v[q]; Qn = -vv * (vv > 0.0 ? Hi[q] : Hi[qn]) / dx; }
    if (cut_w) Qw = 0.0;
    if (cut_e) Qe = 0.0;
    if (cut_s) Qs = 0.0;
    if (cut_n) Qn = 0.0;
    b = max_ref(0.0, Hi[q] + dt * (mb + Qw + Qe + Qs + Qn));
    x0 = b;
  } else {
    const double uw = (i > 0 && !cut_w) ? u[dm.at(j, i - 1)] : 0.0, ue = (i < nx - 1 && !cut_e) ? u[q] : 0.0;
    const double vs = (j > 0 && !cut_s) ? v[dm.at(j - 1, i)] : 0.0, vn = (j < ny - 1 && !cut_n) ? v[q] : 0.0;
    d = 1.0 / dt;
    if (i > 0) d = d - (fs / dx) * min_ref(uw, 0.0);
    if (i < nx - 1) d = d + (fs / dx) * max_ref(ue, 0.0);
    if (j > 0) d = d - (fs / dx) * min_ref(vs, 0.0);
    if (j < ny - 1) d = d + (fs / dx) * max_ref(vn, 0.0);
    if (i > 0) cw = (-fs / dx) * max_ref(uw, 0.0);
    if (i < nx - 1) ce = (fs / dx) * min_ref(ue, 0.0);
    if (j > 0) cs = (-fs / dx) * max_ref(vs, 0.0);
    if (j < ny - 1) cn = (fs / dx) * min_ref(vn, 0.0);
    double r = mb + Hi[q] / dt;
    if (i > 0) r = r + Hi[q] * (1.0 - fs) / dx * min_ref(uw, 0.0) + Hi[qw] * (1.0 - fs) / dx * max_ref(uw, 0.0);
    if (i < nx - 1) r = r - Hi[q] * (1.0 - fs) / dx * max_ref(ue, 0.0) - Hi[qe] * (1.0 - fs) / dx * min_ref(ue, 0.0);
    if (j > 0) r = r + Hi[q] * (1.0 - fs) / dx * min_ref(vs, 0.0) + Hi[qs] * (1.0 - fs) / dx * max_ref(vs, 0.0);
    if (j < ny - 1) r = r - Hi[q] * (1.0 - fs) / dx * max_ref(vn, 0.0) - Hi[qn] * (1.0 - fs) / dx * min_ref(vn, 0.0);
    b = r;
    x0 = Hi[q];
  }
  h.d[q] = d; h.cw[q] = cw; h.ce[q] = ce; h.cs[q] = cs; h.cn[q] = cn; h.b[q] = b; h.x[q] = x0;
}

__device__ __forceinline__ double hsi_apply(const Dims& dm, const HSI& h, const double* x, int j, int i) {
  const long long q = dm.at(j, i);
  double y = h.d[q] * x[q];
  if (i > 0) y = y + h.cw[q] * x[dm.at(j, i - 1)];
  if (i < dm.nx - 1) y = y + h.ce[q] * x[dm.at(j, i + 1)];
  if (j > 0) y = y + h.cs[q] * x[dm.at(j - 1, i)];
  if (j < dm.ny - 1) y = y + h.cn[q] * x[dm.at(j + 1, i)];
  return y;
}

// out = A x (or b - A x when b is given); block partials of (w, out) and (out, out)
__global__ void k_hsi_op(Dims dm, HSI h, const double* x, const double* b, const double* w, double* out,
                         double* part) {
  IDX2D
  double acc[2] = {0.0, 0.0};
  if (j < dm.ny && i < dm.nx) {
    const long long q = dm.at(j, i);
    double y = hsi_apply(dm, h, x, j, i);
    if (b) y = b[q] - y;
    out[q] = y;
    acc[0] = (w ? w[q] : y) * y;
    acc[1] = y * y;
  }
  block_sum<2>(acc);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int blk = blockIdx.y * gridDim.x + blockIdx.x;
    part[2 * blk] = acc[0];
    part[2 * blk + 1] = acc[1];
  }
}

// out = a x + c y + e z (null arrays count as zero); optional division by the diagonal;
// block partials of (w, out) and (out, out)
__global__ void k_hsi_comb(Dims dm, double a, const double* x, double cc, const double* y, double e, const double* z,
                           const double* diag, const double* w, double* out, double* part) {
  IDX2D
  double acc[2] = {0.0, 0.0};
  if (j < dm.ny && i < dm.nx) {
    const long long q = dm.at(j, i);
    double r = a * x[q];
    if (y) r = r + cc * y[q];
    if (z) r = r + e * z[q];
    if (diag) r = r / diag[q];
    out[q] = r;
    acc[0] = (w ? w[q] : r) * r;
    acc[1] = r * r;
  }
  block_sum<2>(acc);
  if (part && threadIdx.x == 0 && threadIdx.y == 0) {
    const int blk = blockIdx.y * gridDim.x + blockIdx.x;
    part[2 * blk] = acc[0];
    part[2 * blk + 1] = acc[1];
  }
}

__global__ void k_hsi_sum(const double* part, int nb, double* out) {
  if (threadIdx.x != 0) return;
  double s0 = 0.0, s1 = 0.0;
  for (int b = 0; b < nb; ++b) {
    s0 += part[2 * b];
    s1 += part[2 * b + 1];
  }
  out[0] = s0;
  out[1] = s1;
}

__global__ void k_hsi_finish(Dims dm, double dt, const double* Hi, const double* x, double* dH, double* Hn) {
  IDX2D
  if (j >= dm.ny || i >= dm.nx) return;
  const long long q = dm.at(j, i);
  Hn[q] = max_ref(0.0, x[q]);
  dH[q] = (Hn[q] - Hi[q]) / dt;
}

}  // namespace

int launch_floating_margin_fraction(Ctx* c) {
  k_float_margin<<<G2T>>>(c->d, c->D(DIVA_F_HI_A), c->I(DIVA_F_MASK_ICE_A), c->I(DIVA_F_MASK_CF_A),
                          c->I(DIVA_F_MASK_SHELF_A), c->D(DIVA_F_FLOAT_MARGIN_FRAC_A), c->D(DIVA_F_HI_EFF_CF_A));
  c->launches++;
  DIVA_LAUNCHED(c, "k_float_margin");
  return DIVA_OK;
}

int launch_thickness_bc(Ctx* c, double dt);

// the two sums of the last reduction, read on the host
static int hsi_read(Ctx* c, int nb, double* s0, double* s1) {
  k_hsi_sum<<<1, 32, 0, c->stream>>>(c->partials, nb, c->scal + SC_TMP0); c->launches++;
  DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal + SC_TMP0, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  *s0 = c->h_scal[0];
  *s1 = c->h_scal[1];
  return DIVA_OK;
}

// calc_dHi_dt_semiimplicit: rows, then BiCGStab with a Jacobi preconditioner to dHi_rtol
static int launch_semiimplicit(Ctx* c, double dt) {
  const Dims d = c->d;
  HSI h;
  h.d = c->kv[KV_X][1]; h.cw = c->kv[KV_B][1]; h.ce = c->kv[KV_R][1]; h.cs = c->kv[KV_RHAT][1];
  h.cn = c->kv[KV_P][1]; h.b = c->kv[KV_PHAT][1]; h.x = c->kv[KV_V][1];
  double *r = c->kv[KV_S][1], *rh = c->kv[KV_SHAT][1], *p = c->kv[KV_T][1];
  double *v = c->kv[KV_X][0], *ph = c->kv[KV_B][0], *s = c->kv[KV_R][0], *sh = c->kv[KV_RHAT][0], *t = c->kv[KV_P][0];
  const dim3 g = grid2d(d.ny, d.nx);
  const int nb = g.x * g.y;
  k_hsi_rows<<<g, block2d(), 0, c->stream>>>(d, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY),
                                             c->D(DIVA_F_SMB_A), c->D(DIVA_F_BMB_A), c->D(DIVA_F_FLOAT_MARGIN_FRAC_A),
                                             c->I(DIVA_F_MASK_ICE_A), c->I(DIVA_F_MASK_SHELF_A),
                                             c->I(DIVA_F_MASK_OCEAN_A), c->I(DIVA_F_MASK_CF_A), h); c->launches++;
  double s0, s1;
  // ||b||, then r = b - A x0 (copied to rhat and p)
  k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, h.b, 0.0, nullptr, 0.0, nullptr, nullptr, nullptr, ph,
                                             c->partials); c->launches++;
  if (int st = hsi_read(c, nb, &s0, &s1)) return st;
  const double target = c->c.dHi_rtol * std::sqrt(s1);
  k_hsi_op<<<g, block2d(), 0, c->stream>>>(d, h, h.x, h.b, nullptr, r, c->partials); c->launches++;
  if (int st = hsi_read(c, nb, &s0, &s1)) return st;
  DIVA_CUDA(c, cudaMemcpyAsync(rh, r, sizeof(double) * d.plane, cudaMemcpyDeviceToDevice, c->stream));
  DIVA_CUDA(c, cudaMemsetAsync(p, 0, sizeof(double) * d.plane, c->stream));
  DIVA_CUDA(c, cudaMemsetAsync(v, 0, sizeof(double) * d.plane, c->stream));
  double rnorm = std::sqrt(s1), rho = 1.0, alpha = 1.0, omega = 1.0;
  int it = 0;
  while (rnorm > target && it < c->c.dHi_maxit) {
    ++it;
    // rho_new = (rhat, r) and p = r + beta (p - omega v); phat = p / diag
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, r, 0.0, nullptr, 0.0, nullptr, nullptr, rh, s, c->partials);
    c->launches++;
    if (int st = hsi_read(c, nb, &s0, &s1)) return st;
    const double rho_new = s0;
    if (!(std::fabs(rho_new) > 0.0) || !std::isfinite(rho_new)) break;
    const double beta = (rho_new / rho) * (alpha / omega);
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, r, beta, p, -beta * omega, v, nullptr, nullptr, p, nullptr);
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, p, 0.0, nullptr, 0.0, nullptr, h.d, nullptr, ph, nullptr);
    k_hsi_op<<<g, block2d(), 0, c->stream>>>(d, h, ph, nullptr, rh, v, c->partials); c->launches += 3;
    if (int st = hsi_read(c, nb, &s0, &s1)) return st;
    alpha = rho_new / s0;
    // s = r - alpha v
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, r, -alpha, v, 0.0, nullptr, nullptr, nullptr, s, c->partials);
    c->launches++;
    if (int st = hsi_read(c, nb, &s0, &s1)) return st;
    if (std::sqrt(s1) <= target) {
      k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, h.x, alpha, ph, 0.0, nullptr, nullptr, nullptr, h.x, nullptr);
      c->launches++;
      rnorm = std::sqrt(s1);
      break;
    }
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, s, 0.0, nullptr, 0.0, nullptr, h.d, nullptr, sh, nullptr);
    k_hsi_op<<<g, block2d(), 0, c->stream>>>(d, h, sh, nullptr, s, t, c->partials); c->launches += 2;
    if (int st = hsi_read(c, nb, &s0, &s1)) return st;
    omega = s1 > 0.0 ? s0 / s1 : 0.0;
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, h.x, alpha, ph, omega, sh, nullptr, nullptr, h.x, nullptr);
    k_hsi_comb<<<g, block2d(), 0, c->stream>>>(d, 1.0, s, -omega, t, 0.0, nullptr, nullptr, nullptr, r, c->partials);
    c->launches += 2;
    if (int st = hsi_read(c, nb, &s0, &s1)) return st;
    rnorm = std::sqrt(s1);
    rho = rho_new;
    if (omega == 0.0) break;
  }
  DIVA_LAUNCHED(c, "semi-implicit thickness solve");
  if (!(rnorm <= target))
    return set_error(c, DIVA_LINEAR_NOT_CONVERGED, "semi-implicit thickness solve did not reach dHi_rtol");
  k_hsi_finish<<<g, block2d(), 0, c->stream>>>(d, dt, c->D(DIVA_F_HI_A), h.x, c->D(DIVA_F_DHI_DT_A),
                                               c->D(DIVA_F_HI_TPLUSDT_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_hsi_finish");
  return DIVA_OK;
}

int launch_calc_dHi_dt(Ctx* c, double dt) {
  const Dims d = c->d;
  if (c->c.choice_ice_integration_method == DIVA_INTEGRATION_SEMIIMPLICIT) {
    if (int st = launch_semiimplicit(c, dt)) return st;
    return launch_thickness_bc(c, dt);
  }
  if (c->c.choice_ice_integration_method == DIVA_INTEGRATION_NONE) {
    DIVA_CUDA(c, cudaMemsetAsync(c->D(DIVA_F_DHI_DT_A), 0, sizeof(double) * d.plane, c->stream));
    return launch_thickness_bc(c, dt);
  }
  double *Qx = c->D(DIVA_F_QX_CX), *Qy = c->D(DIVA_F_QY_CY);
  double *mb = c->quad[0], *rf = c->quad[1];   // scratch planes (grounded-fraction work space)
  k_fluxes<<<G2T>>>(d, dt, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), c->D(DIVA_F_HI_A), Qx, Qy); c->launches++;
  k_cell_budget<<<G2T>>>(d, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_SMB_A), c->D(DIVA_F_BMB_A),
                         c->D(DIVA_F_FLOAT_MARGIN_FRAC_A), c->I(DIVA_F_MASK_CF_A), c->I(DIVA_F_MASK_SHELF_A),
                         c->I(DIVA_F_MASK_OCEAN_A), Qx, Qy, mb, rf); c->launches++;
  k_rescale_faces<<<G2T>>>(d, rf, Qx, Qy); c->launches++;
  k_dhdt<<<G2T>>>(d, dt, c->D(DIVA_F_HI_A), mb, Qx, Qy, c->D(DIVA_F_DHI_DT_A), c->D(DIVA_F_HI_TPLUSDT_A));
  c->launches++;
  return launch_thickness_bc(c, dt);
}

// apply_ice_thickness_BC (:728-931)
int launch_thickness_bc(Ctx* c, double dt) {
  const Dims d = c->d;
  HBC b;
  b.side[0] = c->c.ice_thickness_west_BC;
  b.side[1] = c->c.ice_thickness_east_BC;
  b.side[2] = c->c.ice_thickness_south_BC;
  b.side[3] = c->c.ice_thickness_north_BC;
  b.diva = c->c.choice_ice_dynamics == DIVA_DYN_DIVA;
  k_thickness_bc<<<1, 1024, 0, c->stream>>>(d, b, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_HB_A), c->D(DIVA_F_SL_A),
                                            c->D(DIVA_F_HI_TPLUSDT_A), c->D(DIVA_F_DHI_DT_A)); c->launches++;
  DIVA_LAUNCHED(c, "calc_dHi_dt");
  return DIVA_OK;
}

static int read_scalar(Ctx* c, const double* dev, double* out) {
  DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal, dev, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  *out = c->h_scal[0];
  return DIVA_OK;
}

static int check_hbc(Ctx* c) {
  const int s[4] = {c->c.ice_thickness_west_BC, c->c.ice_thickness_east_BC, c->c.ice_thickness_south_BC,
                    c->c.ice_thickness_north_BC};
  for (int k = 0; k < 4; ++k)
    if (s[k] < DIVA_HBC_ZERO || s[k] > DIVA_HBC_NONE) return set_error(c, DIVA_BAD_INPUT, "ice thickness boundary condition");
  return DIVA_OK;
}

}  // namespace diva

using namespace diva;

extern "C" {

int diva_determine_floating_margin_fraction(diva_ctx_t* h) {
  if (!h) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (int st = launch_floating_margin_fraction(c)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_calc_dHi_dt(diva_ctx_t* h, double dt) {
  if (!h || !(dt > 0.0)) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (int st = check_hbc(c)) return st;
  if (int st = launch_calc_dHi_dt(c, dt)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_calc_critical_timestep_adv(diva_ctx_t* h, double dt_max, double* dt_crit_adv) {
  if (!h || !dt_crit_adv) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const dim3 g = grid2d(c->d.ny, c->d.nx);
  const int nb = g.x * g.y;
  k_crit_adv<<<g, block2d(), 0, c->stream>>>(c->d, 2.0 * dt_max, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY),
                                             c->partials); c->launches++;
  k_extreme_final<<<1, 256, 0, c->stream>>>(c->partials, nb, 2.0 * dt_max, -1, c->scal + SC_TMP0); c->launches++;
  DIVA_LAUNCHED(c, "k_crit_adv");
  double m;
  if (int st = read_scalar(c, c->scal + SC_TMP0, &m)) return st;
  *dt_crit_adv = min_ref(dt_max, m * 0.9);
  return DIVA_OK;
}

int diva_calc_critical_timestep_sia(diva_ctx_t* h, double dt_max, double* dt_crit_sia) {
  if (!h || !dt_crit_sia) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const dim3 g = grid2d(c->d.ny, c->d.nx);
  const int nb = g.x * g.y;
  SiaDt a{c->d, c->zt, dt_max, c->I(DIVA_F_MASK_SHEET_A), c->D(DIVA_F_U_3D_SIA_CX), c->D(DIVA_F_V_3D_SIA_CY),
          c->D(DIVA_F_HI_CX), c->D(DIVA_F_HI_CY), c->D(DIVA_F_DHS_DX_CX), c->D(DIVA_F_DHS_DY_CY),
          c->D(DIVA_F_U_3D_CX), c->D(DIVA_F_V_3D_CY)};
  k_crit_sia<<<g, block2d(), 0, c->stream>>>(a, c->partials); c->launches++;
  k_extreme_final<<<1, 256, 0, c->stream>>>(c->partials, nb, dt_max, -1, c->scal + SC_TMP0); c->launches++;
  DIVA_LAUNCHED(c, "k_crit_sia");
  double m;
  if (int st = read_scalar(c, c->scal + SC_TMP0, &m)) return st;
  *dt_crit_sia = m * 0.9;
  return DIVA_OK;
}

int diva_pc_predictor(diva_ctx_t* h, double dt, double zeta) {
  if (!h || !(dt > 0.0)) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (int st = check_hbc(c)) return st;
  const size_t nb = sizeof(double) * c->d.plane;
  DIVA_CUDA(c, cudaMemcpyAsync(c->D(DIVA_F_DHIDT_HNM1_UNM1), c->D(DIVA_F_DHIDT_HN_UN), nb, cudaMemcpyDeviceToDevice,
                               c->stream));
  if (int st = launch_calc_dHi_dt(c, dt)) return st;
  DIVA_CUDA(c, cudaMemcpyAsync(c->D(DIVA_F_DHIDT_HN_UN), c->D(DIVA_F_DHI_DT_A), nb, cudaMemcpyDeviceToDevice,
                               c->stream));
  k_pc_predict<<<G2T>>>(c->d, dt, zeta, c->D(DIVA_F_HI_A), c->D(DIVA_F_DHIDT_HN_UN), c->D(DIVA_F_DHIDT_HNM1_UNM1),
                        c->D(DIVA_F_HI_PRED), c->D(DIVA_F_HI_OLD)); c->launches++;
  DIVA_LAUNCHED(c, "k_pc_predict");
  if (int st = launch_update_general_ice_model_data(c)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_pc_corrector(diva_ctx_t* h, double dt, double zeta, double eta_min, double* eta) {
  if (!h || !eta || !(dt > 0.0)) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  if (int st = check_hbc(c)) return st;
  const size_t nb = sizeof(double) * c->d.plane;
  if (int st = launch_calc_dHi_dt(c, dt)) return st;
  DIVA_CUDA(c, cudaMemcpyAsync(c->D(DIVA_F_DHIDT_HSTARNP1_UNP1), c->D(DIVA_F_DHI_DT_A), nb, cudaMemcpyDeviceToDevice,
                               c->stream));
  DIVA_CUDA(c, cudaMemcpyAsync(c->D(DIVA_F_HI_A), c->D(DIVA_F_HI_OLD), nb, cudaMemcpyDeviceToDevice, c->stream));
  if (int st = launch_update_general_ice_model_data(c)) return st;
  k_pc_correct<<<G2T>>>(c->d, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_HI_OLD), c->D(DIVA_F_DHIDT_HN_UN),
                        c->D(DIVA_F_DHIDT_HSTARNP1_UNP1), c->D(DIVA_F_HI_CORR), c->D(DIVA_F_DHI_DT_A)); c->launches++;
  const dim3 g = grid2d(c->d.ny, c->d.nx);
  const int nbk = g.x * g.y;
  k_pc_tau<<<g, block2d(), 0, c->stream>>>(c->d, dt, zeta, eta_min, c->D(DIVA_F_HI_CORR), c->D(DIVA_F_HI_PRED),
                                           c->I(DIVA_F_MASK_SHEET_A), c->I(DIVA_F_MASK_GL_A), c->D(DIVA_F_PC_TAU),
                                           c->partials); c->launches++;
  k_extreme_final<<<1, 256, 0, c->stream>>>(c->partials, nbk, eta_min, 1, c->scal + SC_TMP0); c->launches++;
  DIVA_LAUNCHED(c, "pc corrector");
  return read_scalar(c, c->scal + SC_TMP0, eta);
}

int diva_pc_finish(diva_ctx_t* h, double dt) {
  if (!h || !(dt >= 0.0)) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const Dims d = c->d;
  // update_ice_thickness keeps the ice mask of the step for the thermodynamics (:446)
  DIVA_CUDA(c, cudaMemcpyAsync(c->I(DIVA_F_MASK_ICE_A_PREV), c->I(DIVA_F_MASK_ICE_A), sizeof(int) * d.plane,
                               cudaMemcpyDeviceToDevice, c->stream));
  const FixFlags fx{c->c.fixed_shelf_geometry, c->c.fixed_sheet_geometry, c->c.fixed_grounding_line};
  k_pc_finish<<<G2T>>>(d, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_DHI_DT_A), c->D(DIVA_F_HI_TPLUSDT_A), fx,
                       c->I(DIVA_F_MASK_SHELF_A), c->I(DIVA_F_MASK_SHEET_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_pc_finish");
  if (int st = launch_update_general_ice_model_data(c)) return st;
  if (int st = launch_floating_margin_fraction(c)) return st;
  if (c->c.choice_calving_law == DIVA_CALVING_THRESHOLD_THICKNESS) {
    // threshold_thickness_calving (calving_module.f90:62-91), twice so that the calving
    // front may retreat by more than one cell (ice_dynamics_module.f90:562-583)
    for (int pass = 0; pass < 2; ++pass) {
      k_calve_threshold<<<G2T>>>(d, c->I(DIVA_F_MASK_CF_A), c->D(DIVA_F_HI_EFF_CF_A),
                                 c->c.calving_threshold_thickness, c->D(DIVA_F_HI_A)); c->launches++;
      DIVA_LAUNCHED(c, "k_calve_threshold");
      if (int st = launch_update_general_ice_model_data(c)) return st;
      if (pass == 0)
        if (int st = launch_floating_margin_fraction(c)) return st;
    }
  }
  // remove_unconnected_shelves (:932-1044), then the no-ice mask (:586-592)
  int* reach = c->col_flags;   // per-column scratch
  const int* shelf = c->I(DIVA_F_MASK_SHELF_A);
  k_shelf_seed<<<G2T>>>(d, shelf, c->I(DIVA_F_MASK_SHEET_A), reach); c->launches++;
  const dim3 gs((d.ny + kSX - 1) / kSX, (d.nx + kSY - 1) / kSY), bs(kSX, kSY);
  for (long long pass = 0;; ++pass) {
    if (pass > (long long)d.nx * d.ny) return set_error(c, DIVA_TIMEOUT, "remove_unconnected_shelves did not settle");
    DIVA_CUDA(c, cudaMemsetAsync(c->ff_flag, 0, sizeof(int), c->stream));
    k_shelf_spread<<<gs, bs, 0, c->stream>>>(d, shelf, reach, c->ff_flag); c->launches++;
    DIVA_LAUNCHED(c, "k_shelf_spread");
    int changed = 0;
    DIVA_CUDA(c, cudaMemcpyAsync(&changed, c->ff_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
    if (!changed) break;
  }
  const RefGeo rg{c->c.remove_shelves_larger_than_PD, c->c.continental_shelf_calving,
                  c->c.continental_shelf_min_height, c->D(DIVA_F_HI_PD_A), c->D(DIVA_F_HB_PD_A),
                  c->D(DIVA_F_HI_GIAEQ_A), c->D(DIVA_F_HB_GIAEQ_A)};
  k_shelf_remove<<<G2T>>>(d, shelf, reach, c->I(DIVA_F_MASK_NOICE_A), c->c.do_remove_shelves, c->D(DIVA_F_HB_A),
                          c->D(DIVA_F_SL_A), rg, c->D(DIVA_F_HI_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_shelf_remove");
  if (int st = launch_update_general_ice_model_data(c)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

int diva_apply_prescribed_retreat_mask(diva_ctx_t* h, double time, double t0, double t1) {
  if (!h || !(t1 > t0)) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const double wt0 = fmax(0.0, fmin(1.0, (t1 - time) / (t1 - t0)));
  k_retreat_interp<<<G2T>>>(c->d, wt0, c->D(DIVA_F_RETREAT_MASK0_A), c->D(DIVA_F_RETREAT_MASK1_A),
                            c->D(DIVA_F_RETREAT_MASK_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_retreat_interp");
  k_retreat_apply<<<G2T>>>(c->d, c->D(DIVA_F_RETREAT_MASK_A), c->D(DIVA_F_RETREAT_MASK_HI_REF_A),
                           c->D(DIVA_F_HI_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_retreat_apply");
  if (int st = launch_update_general_ice_model_data(c)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

}  // extern "C"
