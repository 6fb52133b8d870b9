// geometry.cu -- the inputs of the velocity solve, on the device.
//
//   update_general_ice_model_data   general_ice_model_data_module.f90:30-86
//     masks + ocean flood-fill      :87-348, :868-988
//   determine_grounded_fractions    :349-783 (CISM bilinear quadrants)
//   calc_pressure_melting_point     thermodynamics_module.f90:609-640
//   calc_ice_rheology               thermodynamics_module.f90:641-753
//   calc_basal_hydrology            basal_conditions_and_sliding_module.f90:90-227
//   driving stress                  ice_velocity_module.f90:288-294
//   set_sico_masks                  ice_velocity_module.f90:1322-1431
//
// This file is compiled with --fmad=false: every product and sum is rounded
// separately, as in the reference, so the masks (which must match bit for bit)
// and the staggered geometry carry no contraction differences.
#include <cfloat>
#include <cmath>
#include <math_constants.h>
#include "ctx.hpp"

namespace diva {
namespace {

__device__ __forceinline__ bool is_floating(double Hi, double Hb, double SL) {
  return Hi < (SL - Hb) * kRhoSW / kRhoI;  // utilities_module.f90:127-137
}

__global__ void k_surface_taf(Dims d, const double* Hi, const double* Hb, const double* SL, double* Hs, double* TAF,
                              int* cand, int* ocean) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double h = Hi[q], b = Hb[q], s = SL[q];
  Hs[q] = h + max_ref(s - kRhoI / kRhoSW * h, b);              // surface_elevation :138-148
  TAF[q] = h - max_ref(0.0, (s - b) * (kRhoSW / kRhoI));       // thickness_above_floatation :149-159
  const int fl = is_floating(h, b, s) ? 1 : 0;
  cand[q] = fl;
  const bool edge = (i == 0 || i == d.nx - 1 || j == 0 || j == d.ny - 1);
  ocean[q] = (fl && edge) ? 1 : 0;
}

// Ocean flood-fill (ocean_floodfill :868-988): the ocean is every floating cell
// 8-connected through floating cells to a floating cell on the domain edge.  The
// reference does a serial stack walk; its result is that connected set, which
// this kernel reaches as the fixed point of a monotone propagation.  Each block
// propagates inside its tile (shared memory, with a one-cell halo read from the
// previous global state) until the tile is stable, then writes back; the host
// relaunches until no block changed anything.
constexpr int kFFX = 32, kFFY = 16;
__global__ void k_floodfill_iter(Dims d, const int* __restrict__ cand, int* ocean, int* changed) {
  __shared__ int so[kFFY + 2][kFFX + 2];
  __shared__ int sc[kFFY + 2][kFFX + 2];
  const int j0 = blockIdx.x * kFFX, i0 = blockIdx.y * kFFY;
  for (int t = threadIdx.y * kFFX + threadIdx.x; t < (kFFX + 2) * (kFFY + 2); t += kFFX * kFFY) {
    const int lj = t % (kFFX + 2), li = t / (kFFX + 2);
    const int j = j0 + lj - 1, i = i0 + li - 1;
    const bool in = (j >= 0 && j < d.ny && i >= 0 && i < d.nx);
    so[li][lj] = in ? ocean[d.at(j, i)] : 0;
    sc[li][lj] = in ? cand[d.at(j, i)] : 0;
  }
  __syncthreads();
  const int lj = threadIdx.x + 1, li = threadIdx.y + 1;
  const int j = j0 + threadIdx.x, i = i0 + threadIdx.y;
  const bool mine = (j < d.ny && i < d.nx);
  int any_change = 0;
  for (int it = 0; it < kFFX * kFFY + 4; ++it) {
    int ch = 0;
    if (mine && sc[li][lj] && !so[li][lj]) {
      if (so[li - 1][lj - 1] | so[li - 1][lj] | so[li - 1][lj + 1] | so[li][lj - 1] | so[li][lj + 1] |
          so[li + 1][lj - 1] | so[li + 1][lj] | so[li + 1][lj + 1]) {
        ch = 1;
      }
    }
    __syncthreads();
    if (ch) so[li][lj] = 1;
    any_change |= ch;
    if (!__syncthreads_or(ch)) break;
  }
  if (mine && any_change) {
    ocean[d.at(j, i)] = 1;
    *changed = 1;
  }
}

__global__ void k_masks_basic(Dims d, const double* Hi, const int* ocean, int floodfill, const int* cand, int* land_o,
                              int* ocean_o, int* ice_o, int* sheet_o, int* shelf_o) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const int oc = floodfill ? ocean[q] : cand[q];
  const int ice = (Hi[q] > DBL_MIN) ? 1 : 0;   // TINY(1._dp)
  land_o[q] = oc ? 0 : 1;
  ocean_o[q] = oc;
  ice_o[q] = ice;
  sheet_o[q] = (ice == 1 && oc == 0) ? 1 : 0;
  shelf_o[q] = (ice == 1 && oc == 1) ? 1 : 0;
}

__global__ void k_masks_transitions(Dims d, const int* land, const int* ocean, const int* ice, const int* sheet,
                                    const int* shelf, int* coast, int* margin, int* gl, int* cf, int* mask) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  int c = 0, m = 0, g = 0, f = 0;
  if (i > 0 && i < d.nx - 1 && j > 0 && j < d.ny - 1) {   // determine_masks_transitions :237-281
    const long long s = d.at(j - 1, i), n = d.at(j + 1, i), w = d.at(j, i - 1), e = d.at(j, i + 1);
    if (land[q] == 1 && ice[q] == 0)
      if (ocean[s] == 1 || ocean[n] == 1 || ocean[w] == 1 || ocean[e] == 1) c = 1;
    if (ice[q] == 1)
      if (ice[s] == 0 || ice[n] == 0 || ice[w] == 0 || ice[e] == 0) m = 1;
    if (sheet[q] == 1)
      if (shelf[s] == 1 || shelf[n] == 1 || shelf[w] == 1 || shelf[e] == 1) g = 1;
    if (ice[q] == 1)
      if ((ocean[s] == 1 && ice[s] == 0) || (ocean[n] == 1 && ice[n] == 0) || (ocean[w] == 1 && ice[w] == 0) ||
          (ocean[e] == 1 && ice[e] == 0))
        f = 1;
  }
  coast[q] = c; margin[q] = m; gl[q] = g; cf[q] = f;
  // determine_masks_total :286-347 (type codes of configuration_module.f90:3171-3179)
  int t = (land[q] == 1) ? 0 : 1;
  if (c == 1) t = 5;
  if (sheet[q] == 1) t = 3;
  else if (shelf[q] == 1) t = 4;
  if (m == 1) t = 6;
  if (g == 1) t = 7;
  if (f == 1) t = 8;
  mask[q] = t;
}

// staggering and slopes of update_general_ice_model_data :60-79
// (map_a_to_cx/cy/b_2D, ddx/ddy_a_to_a/cx/cy_2D of derivatives_and_grids_module.f90)
__global__ void k_stagger_slopes(Dims d, const double* Hi, const double* Hs, const double* Avav, double* Hi_cx,
                                 double* Hi_cy, double* Hi_b, double* Avav_cx, double* Avav_cy, double* dHi_dx,
                                 double* dHi_dy, double* dHs_dx, double* dHs_dy, double* dHs_dx_cx, double* dHs_dy_cx,
                                 double* dHs_dx_cy, double* dHs_dy_cy) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = d.nx, ny = d.ny;
  if (j >= ny || i >= nx) return;
  const double dx = d.dx;
  const long long q = d.at(j, i);
  auto A = [&](const double* f, int jj, int ii) { return f[d.at(jj, ii)]; };
  if (i < nx - 1) {
    Hi_cx[q] = (A(Hi, j, i) + A(Hi, j, i + 1)) / 2.0;
    Avav_cx[q] = (A(Avav, j, i) + A(Avav, j, i + 1)) / 2.0;
    dHs_dx_cx[q] = (A(Hs, j, i + 1) - A(Hs, j, i)) / dx;
    if (j > 0 && j < ny - 1)
      dHs_dy_cx[q] = (A(Hs, j + 1, i) + A(Hs, j + 1, i + 1) - A(Hs, j - 1, i) - A(Hs, j - 1, i + 1)) / (4.0 * dx);
    else if (j == 0)
      dHs_dy_cx[q] = (A(Hs, 1, i) + A(Hs, 1, i + 1) - A(Hs, 0, i) - A(Hs, 0, i + 1)) / (2.0 * dx);
    else
      dHs_dy_cx[q] = (A(Hs, ny - 1, i) + A(Hs, ny - 1, i + 1) - A(Hs, ny - 2, i) - A(Hs, ny - 2, i + 1)) / (2.0 * dx);
  }
  if (j < ny - 1) {
    Hi_cy[q] = (A(Hi, j, i) + A(Hi, j + 1, i)) / 2.0;
    Avav_cy[q] = (A(Avav, j, i) + A(Avav, j + 1, i)) / 2.0;
    dHs_dy_cy[q] = (A(Hs, j + 1, i) - A(Hs, j, i)) / dx;
    if (i > 0 && i < nx - 1)
      dHs_dx_cy[q] = (A(Hs, j, i + 1) + A(Hs, j + 1, i + 1) - A(Hs, j, i - 1) - A(Hs, j + 1, i - 1)) / (4.0 * dx);
    else if (i == 0)
      dHs_dx_cy[q] = (A(Hs, j, 1) + A(Hs, j + 1, 1) - A(Hs, j, 0) - A(Hs, j + 1, 0)) / (2.0 * dx);
    else
      dHs_dx_cy[q] = (A(Hs, j, nx - 1) + A(Hs, j + 1, nx - 1) - A(Hs, j, nx - 2) - A(Hs, j + 1, nx - 2)) / (2.0 * dx);
  }
  if (i < nx - 1 && j < ny - 1)
    Hi_b[q] = (A(Hi, j, i) + A(Hi, j, i + 1) + A(Hi, j + 1, i) + A(Hi, j + 1, i + 1)) / 4.0;
  // ddx_a_to_a_2D / ddy_a_to_a_2D :24-93
  if (i > 0 && i < nx - 1) {
    dHi_dx[q] = (A(Hi, j, i + 1) - A(Hi, j, i - 1)) / (2 * dx);
    dHs_dx[q] = (A(Hs, j, i + 1) - A(Hs, j, i - 1)) / (2 * dx);
  } else if (i == 0) {
    dHi_dx[q] = (A(Hi, j, 1) - A(Hi, j, 0)) / dx;
    dHs_dx[q] = (A(Hs, j, 1) - A(Hs, j, 0)) / dx;
  } else {
    dHi_dx[q] = (A(Hi, j, nx - 1) - A(Hi, j, nx - 2)) / dx;
    dHs_dx[q] = (A(Hs, j, nx - 1) - A(Hs, j, nx - 2)) / dx;
  }
  if (j > 0 && j < ny - 1) {
    dHi_dy[q] = (A(Hi, j + 1, i) - A(Hi, j - 1, i)) / (2 * dx);
    dHs_dy[q] = (A(Hs, j + 1, i) - A(Hs, j - 1, i)) / (2 * dx);
  } else if (j == 0) {
    dHi_dy[q] = (A(Hi, 1, i) - A(Hi, 0, i)) / dx;
    dHs_dy[q] = (A(Hs, 1, i) - A(Hs, 0, i)) / dx;
  } else {
    dHi_dy[q] = (A(Hi, ny - 1, i) - A(Hi, ny - 2, i)) / dx;
    dHs_dy[q] = (A(Hs, ny - 1, i) - A(Hs, ny - 2, i)) / dx;
  }
}

// map_a_to_cx_3D / map_a_to_cy_3D :1513-1578
__global__ void k_stagger3d(Dims d, const double* A, double* Acx, double* Acy) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  for (int k = 0; k < d.nz; ++k) {
    const long long o = (long long)k * d.plane;
    if (i < d.nx - 1) Acx[o + d.at(j, i)] = (A[o + d.at(j, i)] + A[o + d.at(j, i + 1)]) / 2.0;
    if (j < d.ny - 1) Acy[o + d.at(j, i)] = (A[o + d.at(j, i)] + A[o + d.at(j + 1, i)]) / 2.0;
  }
}

// calc_pressure_melting_point :609-640
__global__ void k_pmp(Dims d, Zeta zt, const double* Hi, double* Tp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  for (int k = 0; k < d.nz; ++k) Tp[k * d.plane + q] = kT0 - kCC * Hi[q] * zt.z[k];
}

// calc_ice_rheology :641-738 (A(T), enhancement, vertical average)
__global__ void k_rheology(Dims d, Zeta zt, int choice, int bc_margin, double uniform_A, double m_sheet, double m_shelf,
                           const double* Ti, const int* ice, const int* sheet, const int* shelf, double* A, double* Avav) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const double A_low = 1.14E-05, A_high = 5.47E+10, Q_low = 6.0E+04, Q_high = 13.9E+04;
  const double m = sheet[q] == 1 ? m_sheet : (shelf[q] == 1 ? m_shelf : 1.0);
  const bool apply = sheet[q] == 1 || shelf[q] == 1;
  double prev = 0.0, avg = 0.0;
  for (int k = 0; k < d.nz; ++k) {
    double a;
    if (choice == DIVA_RHEO_UNIFORM) {
      a = uniform_A;
    } else if (ice[q] == 1) {
      const double T = Ti[k * d.plane + q];
      a = (T < 263.15) ? A_low * exp(-Q_low / (kRGas * T)) : A_high * exp(-Q_high / (kRGas * T));
    } else {
      a = bc_margin ? 0.0 : A_low * exp(-Q_low / (kRGas * 263.15));
    }
    if (apply) a = a * m;
    A[k * d.plane + q] = a;
    if (k > 0) avg = avg + 0.5 * (a + prev) * (zt.z[k] - zt.z[k - 1]);  // vertical_average
    prev = a;
  }
  Avav[q] = avg;
}

__global__ void k_stagger2d(Dims d, const double* a, double* cx, double* cy) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  if (i < d.nx - 1) cx[d.at(j, i)] = (a[d.at(j, i)] + a[d.at(j, i + 1)]) / 2.0;
  if (j < d.ny - 1) cy[d.at(j, i)] = (a[d.at(j, i)] + a[d.at(j + 1, i)]) / 2.0;
}

// calc_basal_hydrology :90-143 with the pore-water models :173-227
__global__ void k_basal_hydro(Dims d, int choice, double hb_min, double hb_max, const double* Hi, const double* Hb,
                              const double* SL, double* pwp, double* ob, double* Neff) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  double p;
  if (choice == DIVA_HYDRO_DRY) p = 0.0;
  else if (choice == DIVA_HYDRO_SATURATED) p = -kRhoSW * kGrav * (SL[q] - Hb[q]);
  else {
    const double lam = min_ref(1.0, max_ref(0.0, 1.0 - (Hb[q] - SL[q] - hb_min) / (hb_max - hb_min)));
    p = 0.96 * kRhoI * kGrav * Hi[q] * lam;
  }
  pwp[q] = p;
  const double o = kRhoI * kGrav * Hi[q];
  ob[q] = o;
  Neff[q] = max_ref(0.0, o - p);
}

// calc_fraction_above_zero :521-711 with rotate_quad(_until_match) :712-783
__device__ __forceinline__ void rotate_quad(double& NW, double& NE, double& SW, double& SE) {
  const double f1 = NW, f2 = NE, f3 = SE, f4 = SW;
  NW = f2; NE = f3; SE = f4; SW = f1;
}
__device__ __forceinline__ double nudge(double f, double t) {
  if (f == 0.0) return t;
  if (f > 0.0) return max_ref(t, f);
  if (f < 0.0) return min_ref(-t, f);
  return f;
}
__device__ double fraction_above_zero(double fNW, double fNE, double fSW, double fSE) {
  const double ftol = 1E-4;
  double NW = nudge(fNW, ftol * 1.1), NE = nudge(fNE, ftol * 1.21), SW = nudge(fSW, ftol * 1.13),
         SE = nudge(fSE, ftol * 0.97);
  double phi, aa, bb, cc, dd, x, f1, f2;
  if (NW >= 0.0 && NE >= 0.0 && SW >= 0.0 && SE >= 0.0) {
    phi = 1.0;
  } else if (NW <= 0.0 && NE <= 0.0 && SW <= 0.0 && SE <= 0.0) {
    phi = 0.0;
  } else {
    int scen = 0;
    for (int nit = 1; nit <= 4 && scen == 0; ++nit) {
      rotate_quad(NW, NE, SW, SE);
      if (SW > 0.0 && SE < 0.0 && NE < 0.0 && NW < 0.0) scen = 1;
      else if (SW < 0.0 && SE > 0.0 && NE > 0.0 && NW > 0.0) scen = 2;
      else if (SW > 0.0 && SE > 0.0 && NE < 0.0 && NW < 0.0) scen = 3;
      else if (SW > 0.0 && SE < 0.0 && NE > 0.0 && NW < 0.0) scen = 4;
    }
    if (scen == 1) {
      aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
      phi = ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      if (fabs(dd) < 1E-4) {
        SW = (SW > 0.0) ? SW + 0.1 : SW - 0.1;
        aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
        phi = ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      }
    } else if (scen == 2) {
      aa = -(SW); bb = -(SE - SW); cc = -(NW - SW); dd = -(NE + SW - NW - SE);
      phi = 1.0 - ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      if (fabs(dd) < 1E-4) {
        SW = (SW > 0.0) ? SW + 0.1 : SW - 0.1;
        aa = -(SW); bb = -(SE - SW); cc = -(NW - SW); dd = -(NE + SW - NW - SE);
        phi = 1.0 - ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      }
    } else if (scen == 3) {
      if (fabs(1.0 - NW / NE) < 1E-6 && fabs(1.0 - SW / SE) < 1E-6) {
        phi = SW / (SW - NW);
      } else {
        aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
        x = 0.0; f1 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
        x = 1.0; f2 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
        phi = f2 - f1;
        if (fabs(dd) < 1E-4) {
          SW = (SW > 0.0) ? SW + 0.1 : SW - 0.1;
          aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
          x = 0.0; f1 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
          x = 1.0; f2 = ((bb * cc - aa * dd) * log(fabs(cc + dd * x)) - bb * dd * x) / (dd * dd);
          phi = f2 - f1;
        }
      }
    } else if (scen == 4) {
      aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
      phi = ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
      rotate_quad(NW, NE, SW, SE);
      rotate_quad(NW, NE, SW, SE);
      aa = SW; bb = SE - SW; cc = NW - SW; dd = NE + SW - NW - SE;
      phi = phi + ((bb * cc - aa * dd) * log(fabs(1.0 - (aa * dd) / (bb * cc))) + aa * dd) / (dd * dd);
    } else {
      phi = CUDART_NAN;
    }
  }
  return max_ref(0.0, min_ref(1.0, phi));
}

// determine_grounded_fractions_CISM_quads :420-520 (TAF edge-extended by one cell)
__global__ void k_fgrnd_quads(Dims d, const double* TAF, double* qNW, double* qNE, double* qSW, double* qSE) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  auto T = [&](int jj, int ii) {  // TAF_a_ext(jj+1, ii+1) with the edge copies of :446-455
    jj = jj < 0 ? 0 : (jj > d.ny - 1 ? d.ny - 1 : jj);
    ii = ii < 0 ? 0 : (ii > d.nx - 1 ? d.nx - 1 : ii);
    return TAF[d.at(jj, ii)];
  };
  const double fNW = 0.25 * (T(j + 1, i - 1) + T(j + 1, i) + T(j, i - 1) + T(j, i));
  const double fN = 0.5 * (T(j + 1, i) + T(j, i));
  const double fNE = 0.25 * (T(j + 1, i) + T(j + 1, i + 1) + T(j, i) + T(j, i + 1));
  const double fW = 0.5 * (T(j, i - 1) + T(j, i));
  const double fm = T(j, i);
  const double fE = 0.5 * (T(j, i) + T(j, i + 1));
  const double fSW = 0.25 * (T(j, i - 1) + T(j, i) + T(j - 1, i - 1) + T(j - 1, i));
  const double fS = 0.5 * (T(j, i) + T(j - 1, i));
  const double fSE = 0.25 * (T(j, i) + T(j, i + 1) + T(j - 1, i) + T(j - 1, i + 1));
  const long long q = d.at(j, i);
  qNW[q] = fraction_above_zero(fNW, fN, fW, fm);
  qNE[q] = fraction_above_zero(fN, fNE, fm, fE);
  qSW[q] = fraction_above_zero(fW, fm, fSW, fS);
  qSE[q] = fraction_above_zero(fm, fE, fS, fSE);
}

// determine_grounded_fractions :376-399
__global__ void k_fgrnd_avg(Dims d, const double* qNW, const double* qNE, const double* qSW, const double* qSE,
                            double* fa, double* fcx, double* fcy, double* fb) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  fa[q] = 0.25 * (qNW[q] + qNE[q] + qSW[q] + qSE[q]);
  if (i < d.nx - 1) fcx[q] = 0.25 * (qNE[q] + qSE[q] + qNW[d.at(j, i + 1)] + qSW[d.at(j, i + 1)]);
  if (j < d.ny - 1) fcy[q] = 0.25 * (qNE[q] + qNW[q] + qSE[d.at(j + 1, i)] + qSW[d.at(j + 1, i)]);
  if (i < d.nx - 1 && j < d.ny - 1)
    fb[q] = 0.25 * (qNE[q] + qNW[d.at(j, i + 1)] + qSE[d.at(j + 1, i)] + qSW[d.at(j + 1, i + 1)]);
}

// driving stress, ice_velocity_module.f90:288-294
__global__ void k_taud(Dims d, const double* Hcx, const double* Hcy, const double* sx, const double* sy, double* tx,
                       double* ty) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  if (i < d.nx - 1) tx[q] = -kRhoI * kGrav * Hcx[q] * sx[q];
  if (j < d.ny - 1) ty[q] = -kRhoI * kGrav * Hcy[q] * sy[q];
}

// set_sico_masks :1322-1431.  The reset of DIVA_isfront_inner covers columns
// 1..MIN(ny-1,nx) only (:1384 uses ny where nx is meant); columns beyond keep
// their previous value unless set again, as in the reference.
__global__ void k_sico_masks(Dims d, const double* TAF, const double* Hi, int* combi, int* inner, int* outer) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || i >= d.nx) return;
  const long long q = d.at(j, i);
  const bool fl = TAF[q] < 0.0;
  const double h = Hi[q];
  const int cm = (h == 0.0) ? (fl ? 2 : 1) : (fl ? 3 : 0);
  combi[q] = cm;
  const int ireset = (d.ny - 1 < d.nx) ? d.ny - 1 : d.nx;
  int in = (i < ireset) ? 0 : inner[q];
  const int i1 = i > 0 ? i - 1 : 0, i2 = i < d.nx - 1 ? i + 1 : d.nx - 1;
  const int j1 = j > 0 ? j - 1 : 0, j2 = j < d.ny - 1 ? j + 1 : d.ny - 1;
  const double hw = Hi[d.at(j, i1)], he = Hi[d.at(j, i2)], hs = Hi[d.at(j1, i)], hn = Hi[d.at(j2, i)];
  if (h > 0.0 && (hw == 0.0 || he == 0.0 || hs == 0.0 || hn == 0.0)) in = 1;
  const int out = (h == 0.0 && (hw > 0.0 || he > 0.0 || hs > 0.0 || hn > 0.0)) ? 1 : 0;
  if (in == 1 && cm == 0) in = 0;
  inner[q] = in;
  outer[q] = out;
}

}  // namespace

#define G2 grid2d(c->d.ny, c->d.nx), block2d(), 0, c->stream

int launch_update_general_ice_model_data(Ctx* c) {
  const Dims d = c->d;
  k_surface_taf<<<G2>>>(d, c->D(DIVA_F_HI_A), c->D(DIVA_F_HB_A), c->D(DIVA_F_SL_A), c->D(DIVA_F_HS_A),
                        c->D(DIVA_F_TAF_A), c->ff_ocean + d.plane, c->ff_ocean); c->launches++;
  DIVA_LAUNCHED(c, "k_surface_taf");
  const int* cand = c->ff_ocean + d.plane;
  if (c->c.do_ocean_floodfill) {
    dim3 gb((d.ny + kFFX - 1) / kFFX, (d.nx + kFFY - 1) / kFFY), bb(kFFX, kFFY);
    const long long cap = (long long)d.nx * d.ny + 16;
    long long it = 0;
    for (;;) {
      DIVA_CUDA(c, cudaMemsetAsync(c->ff_flag, 0, sizeof(int), c->stream));
      k_floodfill_iter<<<gb, bb, 0, c->stream>>>(d, cand, c->ff_ocean, c->ff_flag); c->launches++;
      DIVA_LAUNCHED(c, "k_floodfill_iter");
      int h = 0;
      DIVA_CUDA(c, cudaMemcpyAsync(&h, c->ff_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      DIVA_CUDA(c, cudaStreamSynchronize(c->stream));
      if (!h) break;
      if (++it > cap) return set_error(c, DIVA_TIMEOUT, "ocean flood-fill did not settle");
    }
  }
  k_masks_basic<<<G2>>>(d, c->D(DIVA_F_HI_A), c->ff_ocean, c->c.do_ocean_floodfill, cand, c->I(DIVA_F_MASK_LAND_A),
                        c->I(DIVA_F_MASK_OCEAN_A), c->I(DIVA_F_MASK_ICE_A), c->I(DIVA_F_MASK_SHEET_A),
                        c->I(DIVA_F_MASK_SHELF_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_masks_basic");
  k_masks_transitions<<<G2>>>(d, c->I(DIVA_F_MASK_LAND_A), c->I(DIVA_F_MASK_OCEAN_A), c->I(DIVA_F_MASK_ICE_A),
                              c->I(DIVA_F_MASK_SHEET_A), c->I(DIVA_F_MASK_SHELF_A), c->I(DIVA_F_MASK_COAST_A),
                              c->I(DIVA_F_MASK_MARGIN_A), c->I(DIVA_F_MASK_GL_A), c->I(DIVA_F_MASK_CF_A),
                              c->I(DIVA_F_MASK_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_masks_transitions");
  k_stagger_slopes<<<G2>>>(d, c->D(DIVA_F_HI_A), c->D(DIVA_F_HS_A), c->D(DIVA_F_A_FLOW_VAV_A), c->D(DIVA_F_HI_CX),
                           c->D(DIVA_F_HI_CY), c->D(DIVA_F_HI_B), c->D(DIVA_F_A_FLOW_VAV_CX), c->D(DIVA_F_A_FLOW_VAV_CY),
                           c->D(DIVA_F_DHI_DX_A), c->D(DIVA_F_DHI_DY_A), c->D(DIVA_F_DHS_DX_A), c->D(DIVA_F_DHS_DY_A),
                           c->D(DIVA_F_DHS_DX_CX), c->D(DIVA_F_DHS_DY_CX), c->D(DIVA_F_DHS_DX_CY),
                           c->D(DIVA_F_DHS_DY_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_stagger_slopes");
  k_stagger3d<<<G2>>>(d, c->D(DIVA_F_A_FLOW_3D_A), c->D(DIVA_F_A_FLOW_3D_CX), c->D(DIVA_F_A_FLOW_3D_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_stagger3d");
  return DIVA_OK;
}

int launch_pressure_melting_point(Ctx* c) {
  k_pmp<<<G2>>>(c->d, c->zt, c->D(DIVA_F_HI_A), c->D(DIVA_F_TI_PMP_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_pmp");
  return DIVA_OK;
}

int launch_ice_rheology(Ctx* c) {
  if (c->c.choice_ice_rheology != DIVA_RHEO_UNIFORM && c->c.choice_ice_rheology != DIVA_RHEO_HUYBRECHTS1992)
    return set_error(c, DIVA_BAD_INPUT, "unknown choice_ice_rheology");
  k_rheology<<<G2>>>(c->d, c->zt, c->c.choice_ice_rheology, c->c.choice_ice_margin == DIVA_MARGIN_BC,
                     c->c.uniform_flow_factor, c->c.m_enh_sheet, c->c.m_enh_shelf, c->D(DIVA_F_TI_A),
                     c->I(DIVA_F_MASK_ICE_A), c->I(DIVA_F_MASK_SHEET_A), c->I(DIVA_F_MASK_SHELF_A),
                     c->D(DIVA_F_A_FLOW_3D_A), c->D(DIVA_F_A_FLOW_VAV_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_rheology");
  k_stagger3d<<<G2>>>(c->d, c->D(DIVA_F_A_FLOW_3D_A), c->D(DIVA_F_A_FLOW_3D_CX), c->D(DIVA_F_A_FLOW_3D_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_stagger3d");
  k_stagger2d<<<G2>>>(c->d, c->D(DIVA_F_A_FLOW_VAV_A), c->D(DIVA_F_A_FLOW_VAV_CX), c->D(DIVA_F_A_FLOW_VAV_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_stagger2d");
  return DIVA_OK;
}

int launch_basal_conditions(Ctx* c) {
  k_basal_hydro<<<G2>>>(c->d, c->c.choice_basal_hydrology, c->c.Martin2011_hydro_Hb_min, c->c.Martin2011_hydro_Hb_max,
                        c->D(DIVA_F_HI_A), c->D(DIVA_F_HB_A), c->D(DIVA_F_SL_A), c->D(DIVA_F_PORE_WATER_PRESSURE_A),
                        c->D(DIVA_F_OVERBURDEN_PRESSURE_A), c->D(DIVA_F_NEFF_A)); c->launches++;
  DIVA_LAUNCHED(c, "k_basal_hydro");
  return DIVA_OK;
}

int launch_grounded_fractions(Ctx* c) {
  k_fgrnd_quads<<<G2>>>(c->d, c->D(DIVA_F_TAF_A), c->quad[0], c->quad[1], c->quad[2], c->quad[3]); c->launches++;
  DIVA_LAUNCHED(c, "k_fgrnd_quads");
  k_fgrnd_avg<<<G2>>>(c->d, c->quad[0], c->quad[1], c->quad[2], c->quad[3], c->D(DIVA_F_F_GRND_A),
                      c->D(DIVA_F_F_GRND_CX), c->D(DIVA_F_F_GRND_CY), c->D(DIVA_F_F_GRND_B)); c->launches++;
  DIVA_LAUNCHED(c, "k_fgrnd_avg");
  return DIVA_OK;
}

int launch_driving_stress(Ctx* c) {
  k_taud<<<G2>>>(c->d, c->D(DIVA_F_HI_CX), c->D(DIVA_F_HI_CY), c->D(DIVA_F_DHS_DX_CX), c->D(DIVA_F_DHS_DY_CY),
                 c->D(DIVA_F_TAUDX_CX), c->D(DIVA_F_TAUDY_CY)); c->launches++;
  DIVA_LAUNCHED(c, "k_taud");
  return DIVA_OK;
}

int launch_sico_masks(Ctx* c) {
  k_sico_masks<<<G2>>>(c->d, c->D(DIVA_F_TAF_A), c->D(DIVA_F_HI_A), c->I(DIVA_F_DIVA_MASK_COMBI),
                       c->I(DIVA_F_DIVA_ISFRONT_INNER), c->I(DIVA_F_DIVA_ISFRONT_OUTER)); c->launches++;
  DIVA_LAUNCHED(c, "k_sico_masks");
  return DIVA_OK;
}

}  // namespace diva
