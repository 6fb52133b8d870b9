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

__global__ void k_pc_finish(Dims d, double dt, double* Hi, const double* dH, double* Hn) {
  IDX2D
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  Hn[q] = max_ref(0.0, Hi[q] + dt * dH[q]);
  Hi[q] = max_ref(0.0, Hn[q]);
}

}  // namespace

int launch_floating_margin_fraction(Ctx* c) {
  k_float_margin<<<G2T>>>(c->d, c->D(DIVA_F_HI_A), c->I(DIVA_F_MASK_ICE_A), c->I(DIVA_F_MASK_CF_A),
                          c->I(DIVA_F_MASK_SHELF_A), c->D(DIVA_F_FLOAT_MARGIN_FRAC_A), c->D(DIVA_F_HI_EFF_CF_A));
  c->launches++;
  DIVA_LAUNCHED(c, "k_float_margin");
  return DIVA_OK;
}

int launch_calc_dHi_dt(Ctx* c, double dt) {
  const Dims d = c->d;
  double *Qx = c->D(DIVA_F_QX_CX), *Qy = c->D(DIVA_F_QY_CY);
  double *mb = c->quad[0], *rf = c->quad[1];   // scratch planes (grounded-fraction work space)
  k_fluxes<<<G2T>>>(d, dt, c->D(DIVA_F_U_VAV_CX), c->D(DIVA_F_V_VAV_CY), c->D(DIVA_F_HI_A), Qx, Qy); c->launches++;
  k_cell_budget<<<G2T>>>(d, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_SMB_A), c->D(DIVA_F_BMB_A),
                         c->D(DIVA_F_FLOAT_MARGIN_FRAC_A), c->I(DIVA_F_MASK_CF_A), c->I(DIVA_F_MASK_SHELF_A),
                         c->I(DIVA_F_MASK_OCEAN_A), Qx, Qy, mb, rf); c->launches++;
  k_rescale_faces<<<G2T>>>(d, rf, Qx, Qy); c->launches++;
  k_dhdt<<<G2T>>>(d, dt, c->D(DIVA_F_HI_A), mb, Qx, Qy, c->D(DIVA_F_DHI_DT_A), c->D(DIVA_F_HI_TPLUSDT_A));
  c->launches++;
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
  // update_ice_thickness keeps the ice mask of the step for the thermodynamics (:446)
  DIVA_CUDA(c, cudaMemcpyAsync(c->I(DIVA_F_MASK_ICE_A_PREV), c->I(DIVA_F_MASK_ICE_A), sizeof(int) * c->d.plane,
                               cudaMemcpyDeviceToDevice, c->stream));
  k_pc_finish<<<G2T>>>(c->d, dt, c->D(DIVA_F_HI_A), c->D(DIVA_F_DHI_DT_A), c->D(DIVA_F_HI_TPLUSDT_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_pc_finish");
  if (int st = launch_update_general_ice_model_data(c)) return st;
  if (int st = launch_floating_margin_fraction(c)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}

}  // extern "C"
