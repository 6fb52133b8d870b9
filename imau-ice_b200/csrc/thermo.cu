// thermo.cu -- run_thermo_model with the 3D heat equation (thermodynamics_module.f90:
// 29-608, derivatives_and_grids_module.f90:1892-2061) on the device: one thread per
// grid column assembles the column's implicit system over C%dt_thermo (vertical
// diffusion, vertical and upwind horizontal advection, strain heating, the surface,
// shelf-base and geothermal/frictional bed conditions) and solves it in registers.
//
// The column solve is Gaussian elimination with partial pivoting in the order of
// LAPACK's dgtsv (the routine the reference's tridiagonal_solve calls); compiled
// without FMA contraction so that every column is the oracle's sequence of IEEE
// operations (exp and erf aside, which are the CUDA library's).
#include <cmath>
#include "ctx.hpp"

namespace diva {
namespace {

constexpr double kSecPerYear = 31556943.36;   // parameters_module.f90:12

#define IDX2D                                                            \
  const int j = blockIdx.x * blockDim.x + threadIdx.x;                   \
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
#define G2H grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream

struct ThermoArgs {
  Dims d;
  Zeta zt;
  double dt, T_ocean;        // the shelf-base ocean temperature with ocean model 'none'
  int ocean_input;           // 1: T_ocean_base_a (deg C) instead
  const double* To_in;
  int heatcap, conduct;
  double cp_uniform, k_uniform;
  int no_friction;
  // inputs and state
  const double *Hi, *Hs, *Ts, *ghf, *dHi_dt, *dHb_dt, *dHs_dx, *dHs_dy, *dHi_dx, *dHi_dy, *Tp;
  const double *u3, *v3, *w3, *ucx, *vcy, *beta, *ub, *vb, *uvav, *vvav, *smb;
  const int *ice, *prev, *sheet, *shelf;
  double *Ti, *Tn, *Cp, *Ki, *fh, *dHs_dt, *zdt, *zdx, *zdy, *zdz;
  int* unstable;
};

// newly ice-covered columns take the temperature of an upwind ice neighbour (:46-72)
__global__ void k_new_ice(ThermoArgs a) {
  IDX2D
  const Dims& d = a.d;
  if (j < 1 || j > d.ny - 2 || i < 1 || i > d.nx - 2) return;
  const long long q = d.at(j, i);
  if (!(a.ice[q] == 1 && a.prev[q] == 0)) return;
  long long s = -1;
  if (a.uvav[d.at(j, i - 1)] > 0.0 && a.prev[d.at(j, i - 1)] == 1) s = d.at(j, i - 1);
  else if (a.uvav[q] < 0.0 && a.prev[d.at(j, i + 1)] == 1) s = d.at(j, i + 1);
  else if (a.vvav[d.at(j - 1, i)] > 0.0 && a.prev[d.at(j - 1, i)] == 1) s = d.at(j - 1, i);
  else if (a.vvav[q] < 0.0 && a.prev[d.at(j + 1, i)] == 1) s = d.at(j + 1, i);
  for (int k = 0; k < d.nz; ++k) a.Ti[k * d.plane + q] = s >= 0 ? a.Ti[k * d.plane + s] : min_ref(a.Ts[q], kT0);
}

// frictional heating (:484-522), heat capacity (:523-565), conductivity (:566-608)
__global__ void k_thermo_props(ThermoArgs a) {
  IDX2D
  const Dims& d = a.d;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (a.no_friction) a.fh[q] = 0.0;
  else if (j >= 1 && j <= d.ny - 2 && i >= 1 && i <= d.nx - 2)
    a.fh[q] = a.sheet[q] == 1 ? a.beta[q] * (a.ub[q] * a.ub[q] + a.vb[q] * a.vb[q]) : 0.0;
  for (int k = 0; k < d.nz; ++k) {
    const long long p = k * d.plane + q;
    a.Cp[p] = a.heatcap == DIVA_HEATCAP_UNIFORM ? a.cp_uniform : 2115.3 + 7.79293 * (a.Ti[p] - kT0);
    a.Ki[p] = a.conduct == DIVA_CONDUCT_UNIFORM ? a.k_uniform : 3.101E+08 * exp(-0.0057 * a.Ti[p]);
  }
}

// dHs_dt, calculate_zeta_derivatives (:1892-1929) and the surface layer (:189-193)
__global__ void k_heat_prep(ThermoArgs a) {
  IDX2D
  const Dims& d = a.d;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double hs = a.shelf[q] == 0 ? a.dHi_dt[q] + a.dHb_dt[q] : a.dHi_dt[q] * (1.0 - kRhoI / kRhoSW);
  a.dHs_dt[q] = hs;
  const double inv = 1.0 / a.Hi[q];
  a.zdz[q] = -inv;
  for (int k = 0; k < d.nz; ++k) {
    const long long p = k * d.plane + q;
    const double z = a.zt.z[k];
    a.zdt[p] = inv * (hs - z * a.dHi_dt[q]);
    a.zdx[p] = inv * (a.dHs_dx[q] - z * a.dHi_dx[q]);
    a.zdy[p] = inv * (a.dHs_dy[q] - z * a.dHi_dy[q]);
  }
  a.Ti[q] = min_ref(kT0, a.Ts[q]);
}

// the dgtsv elimination (see the oracle's orc_tridiagonal_solve); 0 or the failing row + 1
__device__ int tridiagonal_solve(int n, double* dl, double* d, double* du, double* b) {
  for (int i = 0; i < n - 1; ++i) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] == 0.0) return i + 1;
      const double fact = dl[i] / d[i];
      d[i + 1] = d[i + 1] - fact * du[i];
      b[i + 1] = b[i + 1] - fact * b[i];
      if (i < n - 2) dl[i] = 0.0;
    } else {
      const double fact = d[i] / dl[i];
      d[i] = dl[i];
      const double t = d[i + 1];
      d[i + 1] = du[i] - fact * t;
      if (i < n - 2) {
        dl[i] = du[i + 1];
        du[i + 1] = -fact * dl[i];
      }
      du[i] = t;
      const double tb = b[i];
      b[i] = b[i + 1];
      b[i + 1] = tb - fact * b[i + 1];
    }
  }
  if (d[n - 1] == 0.0) return n;
  b[n - 1] = b[n - 1] / d[n - 1];
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
  for (int i = n - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - dl[i] * b[i + 2]) / d[i];
  return 0;
}

// one column of solve_3D_heat_equation (:214-330)
__global__ void k_heat_columns(ThermoArgs a) {
  IDX2D
  const Dims& d = a.d;
  if (j < 1 || j > d.ny - 2 || i < 1 || i > d.nx - 2) return;
  const long long q = d.at(j, i);
  const int nz = d.nz;
  const long long P = d.plane;
  a.unstable[q] = 0;
  if (a.ice[q] == 0) {
    for (int k = 0; k < nz; ++k) a.Tn[k * P + q] = a.Ti[q];
    return;
  }
  if (a.Hi[q] < 1.0) {
    for (int k = 0; k < nz; ++k) a.Tn[k * P + q] = min_ref(kT0, a.Ts[q]);
    return;
  }
  double dl[kMaxNz], dg[kMaxNz], du[kMaxNz], b[kMaxNz];
  const double* z = a.zt.z;
  const double zdz = a.zdz[q], dx = d.dx, dt = a.dt;
  for (int k = 1; k < nz - 1; ++k) {
    const long long p = k * P + q;
    const double ak = z[k] - z[k - 1], bk = z[k + 1] - z[k];
    const double ca = -bk / (ak * (ak + bk)), cb = (bk - ak) / (ak * bk), cc = ak / (bk * (ak + bk));
    const double caa = 2.0 / (ak * (ak + bk)), cbb = -2.0 / (ak * bk), ccc = 2.0 / (bk * (ak + bk));
    double heat = 0.0;
    if (a.sheet[q] == 1)
      heat = ((-kGrav * z[k]) / a.Cp[p]) *
             ((ca * a.u3[p - P] + cb * a.u3[p] + cc * a.u3[p + P]) * a.dHs_dx[q] +
              (ca * a.v3[p - P] + cb * a.v3[p] + cc * a.v3[p + P]) * a.dHs_dy[q]);
    double udx, vdy;
    if (a.u3[p] > 0.0) udx = a.ucx[k * P + d.at(j, i - 1)] * (a.Ti[p] - a.Ti[k * P + d.at(j, i - 1)]) / dx;
    else udx = a.ucx[p] * (a.Ti[k * P + d.at(j, i + 1)] - a.Ti[p]) / dx;
    if (a.v3[p] > 0.0) vdy = a.vcy[k * P + d.at(j - 1, i)] * (a.Ti[p] - a.Ti[k * P + d.at(j - 1, i)]) / dx;
    else vdy = a.vcy[p] * (a.Ti[k * P + d.at(j + 1, i)] - a.Ti[p]) / dx;
    const double f1 = (a.Ki[p] * (zdz * zdz)) / (kRhoI * a.Cp[p]);
    const double f2 = a.zdt[p] + a.zdx[p] * a.u3[p] + a.zdy[p] * a.v3[p] + zdz * a.w3[p];
    const double f3 = heat + (udx + vdy) - a.Ti[p] / dt;
    dl[k - 1] = f1 * caa - f2 * ca;
    dg[k] = f1 * cbb - f2 * cb - 1.0 / dt;
    du[k] = f1 * ccc - f2 * cc;
    b[k] = f3;
  }
  dg[0] = 1.0;
  du[0] = 0.0;
  b[0] = min_ref(kT0, a.Ts[q]);
  const long long pb = (long long)(nz - 1) * P + q;
  const double bed = (z[nz - 1] - z[nz - 2]) * (a.ghf[q] + a.fh[q]) / (zdz * a.Ki[pb]);
  if (a.shelf[q] == 1) {
    const double To = a.ocean_input ? a.To_in[q] + kT0 : a.T_ocean;
    dl[nz - 2] = 0.0;
    dg[nz - 1] = 1.0;
    b[nz - 1] = min_ref(kT0, min_ref(a.Tp[pb], To));
  } else if (a.Ti[pb] >= a.Tp[pb]) {
    dl[nz - 2] = 0.0;
    dg[nz - 1] = 1.0;
    b[nz - 1] = a.Tp[pb];
  } else {
    dl[nz - 2] = 1.0;
    dg[nz - 1] = -1.0;
    b[nz - 1] = bed;
  }
  const int info = tridiagonal_solve(nz, dl, dg, du, b);
  bool bad = false;
  double mn = INFINITY;
  for (int k = 0; k < nz; ++k) {
    double t = info ? NAN : b[k];
    if (k < nz - 1) t = min_ref(t, a.Tp[k * P + q]);
    else if (t >= a.Tp[pb]) t = min_ref(a.Tp[pb], a.Ti[(long long)(nz - 2) * P + q] - bed);
    a.Tn[k * P + q] = t;
    if (t != t) bad = true;
    mn = min_ref(mn, t);
  }
  if (mn < 150.0 || bad) a.unstable[q] = 1;
}

// Neumann_BC_a_3D (:2034-2061): the first and last rows, then the first and last columns
__global__ void k_neumann_rows(Dims d, double* T) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (i >= d.nx) return;
  T[k * d.plane + d.at(0, i)] = T[k * d.plane + d.at(1, i)];
  T[k * d.plane + d.at(d.ny - 1, i)] = T[k * d.plane + d.at(d.ny - 2, i)];
}
__global__ void k_neumann_cols(Dims d, double* T) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (j >= d.ny) return;
  T[k * d.plane + d.at(j, 0)] = T[k * d.plane + d.at(j, 1)];
  T[k * d.plane + d.at(j, d.nx - 1)] = T[k * d.plane + d.at(j, d.nx - 2)];
}

__global__ void k_count_unstable(Dims d, const int* flag, double* part) {
  IDX2D
  double v[1] = {0.0};
  if (j >= 1 && j <= d.ny - 2 && i >= 1 && i <= d.nx - 2) v[0] = flag[d.at(j, i)];
  block_sum<1>(v);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = v[0];
}
__global__ void k_sum_final(const double* part, int nb, double* out) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nb; ++b) s += part[b];
  *out = s;
}

// replace_Ti_with_robin_solution (:384-481) for the flagged columns
__global__ void k_robin(ThermoArgs a) {
  IDX2D
  const Dims& d = a.d;
  if (j < 1 || j > d.ny - 2 || i < 1 || i > d.nx - 2) return;
  const long long q = d.at(j, i);
  if (!a.unstable[q]) return;
  const long long P = d.plane;
  const double* z = a.zt.z;
  const double K = 9.828 * kSecPerYear * exp(-0.0057 * kT0);
  const double kappa = K / (kRhoI * 2127.5);
  const double grad = -a.ghf[q] / K;
  const double Ts = min_ref(kT0, a.Ts[q]), Hi = a.Hi[q];
  if (a.sheet[q] == 1) {
    if (a.smb[q] > 0.0) {
      const double L = sqrt(2.0 * kappa * Hi / a.smb[q]);
      for (int k = 0; k < d.nz; ++k) {
        const double erf1 = erf((1.0 - z[k]) * Hi / L), erf2 = erf(Hi / L);
        a.Tn[k * P + q] = Ts + sqrt(kPi) / 2.0 * L * grad * (erf1 - erf2);
      }
    } else {
      for (int k = 0; k < d.nz; ++k) a.Tn[k * P + q] = Ts + ((kT0 - kCC * Hi) - Ts) * z[k];
    }
  } else if (a.shelf[q] == 1) {
    // the Robin profile adds T0 to its ocean temperature, which with ocean model 'none' is
    // already T0 + T_ocean_mean_PD_ANT (:455-465, as written)
    const double To = a.ocean_input ? a.To_in[q] : a.T_ocean;
    for (int k = 0; k < d.nz; ++k) a.Tn[k * P + q] = Ts + z[k] * (kT0 + To - Ts);
  } else {
    for (int k = 0; k < d.nz; ++k) a.Tn[k * P + q] = Ts;
  }
  for (int k = 0; k < d.nz; ++k) a.Tn[k * P + q] = min_ref(a.Tn[k * P + q], a.Tp[k * P + q]);
}

}  // namespace
}  // namespace diva

using namespace diva;

extern "C" int diva_run_thermo_model(diva_ctx_t* h, int32_t do_solve, int32_t* n_unstable) {
  if (!h || !n_unstable) return DIVA_BAD_INPUT;
  Ctx* c = &h->c;
  const Dims d = c->d;
  *n_unstable = 0;
  if (do_solve && !(c->c.dt_thermo > 0.0)) return set_error(c, DIVA_BAD_INPUT, "dt_thermo must be > 0");
  if (d.nz > kMaxNz) return set_error(c, DIVA_BAD_INPUT, "nz");
  ThermoArgs a;
  a.d = d;
  a.zt = c->zt;
  a.dt = c->c.dt_thermo;
  a.T_ocean = kT0 + c->c.T_ocean_mean_PD_ANT;
  a.ocean_input = c->c.ocean_temperature_input;
  a.To_in = c->D(DIVA_F_T_OCEAN_BASE_A);
  a.heatcap = c->c.choice_ice_heat_capacity;
  a.conduct = c->c.choice_ice_thermal_conductivity;
  a.cp_uniform = c->c.uniform_ice_heat_capacity;
  a.k_uniform = c->c.uniform_ice_thermal_conductivity;
  a.no_friction = c->c.choice_ice_dynamics == DIVA_DYN_SIA || c->c.choice_sliding_law == DIVA_SLIDING_NONE;
  a.Hi = c->D(DIVA_F_HI_A); a.Hs = c->D(DIVA_F_HS_A); a.Ts = c->D(DIVA_F_T_SURF_ANNUAL_A); a.ghf = c->D(DIVA_F_GHF_A);
  a.dHi_dt = c->D(DIVA_F_DHI_DT_A); a.dHb_dt = c->D(DIVA_F_DHB_DT_A);
  a.dHs_dx = c->D(DIVA_F_DHS_DX_A); a.dHs_dy = c->D(DIVA_F_DHS_DY_A);
  a.dHi_dx = c->D(DIVA_F_DHI_DX_A); a.dHi_dy = c->D(DIVA_F_DHI_DY_A); a.Tp = c->D(DIVA_F_TI_PMP_A);
  a.u3 = c->D(DIVA_F_U_3D_A); a.v3 = c->D(DIVA_F_V_3D_A); a.w3 = c->D(DIVA_F_W_3D_A);
  a.ucx = c->D(DIVA_F_U_3D_CX); a.vcy = c->D(DIVA_F_V_3D_CY);
  a.beta = c->D(DIVA_F_BETA_A); a.ub = c->D(DIVA_F_U_BASE_A); a.vb = c->D(DIVA_F_V_BASE_A);
  a.uvav = c->D(DIVA_F_U_VAV_CX); a.vvav = c->D(DIVA_F_V_VAV_CY); a.smb = c->D(DIVA_F_SMB_A);
  a.ice = c->I(DIVA_F_MASK_ICE_A); a.prev = c->I(DIVA_F_MASK_ICE_A_PREV);
  a.sheet = c->I(DIVA_F_MASK_SHEET_A); a.shelf = c->I(DIVA_F_MASK_SHELF_A);
  a.Ti = c->D(DIVA_F_TI_A); a.Tn = c->staging; a.Cp = c->D(DIVA_F_CPI_A); a.Ki = c->D(DIVA_F_KI_A);
  a.fh = c->D(DIVA_F_FRICTIONAL_HEATING_A); a.dHs_dt = c->D(DIVA_F_DHS_DT_A);
  a.zdt = c->D(DIVA_F_DZETA_DT_A); a.zdx = c->D(DIVA_F_DZETA_DX_A); a.zdy = c->D(DIVA_F_DZETA_DY_A);
  a.zdz = c->D(DIVA_F_DZETA_DZ_A);
  a.unstable = c->col_flags;   // per-column scratch (free outside the viscosity iteration)
  k_new_ice<<<G2H>>>(a); c->launches++;
  k_thermo_props<<<G2H>>>(a); c->launches++;
  DIVA_LAUNCHED(c, "k_thermo_props");
  if (int st = launch_pressure_melting_point(c)) return st;
  if (do_solve) {
    k_heat_prep<<<G2H>>>(a); c->launches++;
    k_heat_columns<<<G2H>>>(a); c->launches++;
    k_neumann_rows<<<dim3((d.nx + 127) / 128, d.nz), 128, 0, c->stream>>>(d, c->staging); c->launches++;
    k_neumann_cols<<<dim3((d.ny + 127) / 128, d.nz), 128, 0, c->stream>>>(d, c->staging); c->launches++;
    const dim3 g = grid2d(d.ny, d.nx);
    const int nb = g.x * g.y;
    k_count_unstable<<<g, block2d(), 0, c->stream>>>(d, c->col_flags, c->partials); c->launches++;
    k_sum_final<<<1, 32, 0, c->stream>>>(c->partials, nb, c->scal + SC_TMP0); c->launches++;
    DIVA_LAUNCHED(c, "solve_3D_heat_equation");
    DIVA_CUDA(c, cudaMemcpyAsync(c->h_scal, c->scal + SC_TMP0, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
    const int nu = (int)c->h_scal[0];
    const int limit = (int)std::ceil((double)(d.nx * d.ny) / 100.0);
    if (nu >= limit) return set_error(c, DIVA_NAN_DETECTED, "heat equation solver unstable for more than 1% of grid cells");
    *n_unstable = nu;
    if (nu > 0) {
      k_robin<<<G2H>>>(a); c->launches++;
      DIVA_LAUNCHED(c, "k_robin");
    }
    DIVA_CUDA(c, cudaMemcpyAsync(a.Ti, c->staging, sizeof(double) * d.nz * d.plane, cudaMemcpyDeviceToDevice,
                                 c->stream));
  }
  if (int st = launch_ice_rheology(c)) return st;
  DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
  return DIVA_OK;
}
