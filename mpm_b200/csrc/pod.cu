// pod.cu -- packing of the device particle state into the reference's
// PODParticle records (Particle::pod, particle.tcc:180-306; record layout
// pod_particle.h:12-62 and the field table of pod_particle.cc) for the HDF5
// particle table (Mesh::write_particles_hdf5, mesh.tcc:1573-1613).
//
// The record layout is the caller's: byte offset and size of each of the 74
// fields, as the reference passes them to H5TBmake_table.  One thread writes
// one field of one record, so consecutive threads write neighbouring bytes of
// a record.
#include <cuda_runtime.h>

#include "mpm_kernels.h"
#include "mpm_state.cuh"

namespace mpm_b200 {
namespace {

template <int DIM, bool MIXED>
__device__ __forceinline__ double pf_value(const DevState& s, int f, int c, int64_t p) {
  // FP64 layout offset f + component c, read from whichever buffer holds it
  const int64_t np = s.np;
  if constexpr (!MIXED) {
    return s.pf[(int64_t)(f + c) * np + p];
  } else {
    if (f == PF<DIM>::X) return s.pf[(int64_t)(PDX<DIM>::X + c) * np + p];
    if (f == PF<DIM>::U) return s.pf[(int64_t)(PDX<DIM>::U + c) * np + p];
    const float* m = s.pm;
    if (f == PF<DIM>::V) return (double)m[(int64_t)(PM<DIM>::V + c) * np + p];
    if (f == PF<DIM>::S) return (double)m[(int64_t)(PM<DIM>::S + c) * np + p];
    if (f == PF<DIM>::E) return (double)m[(int64_t)(PM<DIM>::E + c) * np + p];
    if (f == PF<DIM>::F) {
      const bool diag = DIM == 2 ? (c == 0 || c == 3) : (c % 4 == 0);
      return (double)m[(int64_t)(PM<DIM>::H + c) * np + p] + (diag ? 1.0 : 0.0);
    }
    const double jp = (double)m[(int64_t)PM<DIM>::JP * np + p];
    if (f == PF<DIM>::VOL) return (double)m[(int64_t)PM<DIM>::V0 * np + p] * (1.0 + jp);
    if (f == PF<DIM>::RHO) return (double)m[(int64_t)PM<DIM>::RHO0 * np + p] / (1.0 + jp);
    return (double)m[(int64_t)PM<DIM>::MASS * np + p];  // MASS
  }
}

template <int DIM, bool MIXED>
__device__ __forceinline__ double svar_value(const DevState& s, int k, int64_t p) {
  const int64_t np = s.np;
  if constexpr (!MIXED) {
    return s.sv[(int64_t)k * np + p];
  } else {
    if (k == SV_PD) return s.pf[(int64_t)PDX<DIM>::PDS * np + p];
    return (double)s.svf[(int64_t)k * np + p];
  }
}

// Value of field f (PODParticle order) of particle p; kind: 0 double,
// 1 unsigned 64-bit, 2 unsigned 32-bit, 3 bool.
template <int DIM, bool MIXED>
__device__ void pod_field(const DevState& s, const PodAux& a, int f, int64_t p, double& dv,
                          uint64_t& uv, int& kind) {
  kind = 0;
  dv = 0.0;
  uv = 0;
  const int64_t np = s.np;
  auto vec3 = [&](int off, int c) { return c < DIM ? pf_value<DIM, MIXED>(s, off, c, p) : 0.0; };
  if (f == 0) {  // id
    kind = 1;
    uv = a.id[p];
  } else if (f == 1) {
    dv = pf_value<DIM, MIXED>(s, PF<DIM>::MASS, 0, p);
  } else if (f == 2) {
    dv = pf_value<DIM, MIXED>(s, PF<DIM>::VOL, 0, p);
  } else if (f == 3) {  // pressure: not a state variable of LinearElastic / MohrCoulomb
    dv = 0.0;
  } else if (f < 7) {
    dv = vec3(PF<DIM>::X, f - 4);
  } else if (f < 10) {
    dv = vec3(PF<DIM>::U, f - 7);
  } else if (f < 13) {
    dv = a.nsize[(int64_t)(f - 10) * np + p];
  } else if (f < 16) {
    dv = vec3(PF<DIM>::V, f - 13);
  } else if (f < 19) {
    dv = a.acc[(int64_t)(f - 16) * np + p];
  } else if (f < 25) {  // stress xx yy zz xy yz xz
    const int k = f - 19;
    dv = k < PF<DIM>::NS ? pf_value<DIM, MIXED>(s, PF<DIM>::S, k, p) : 0.0;
  } else if (f < 31) {  // strain xx yy zz xy yz xz (2D stores xx yy xy)
    const int k = f - 25;
    if constexpr (DIM == 3) {
      dv = pf_value<DIM, MIXED>(s, PF<3>::E, k, p);
    } else {
      dv = k == 0 ? pf_value<DIM, MIXED>(s, PF<2>::E, 0, p)
                  : (k == 1 ? pf_value<DIM, MIXED>(s, PF<2>::E, 1, p)
                            : (k == 3 ? pf_value<DIM, MIXED>(s, PF<2>::E, 2, p) : 0.0));
    }
  } else if (f < 40) {  // deformation gradient, row major 3x3
    const int r = (f - 31) / 3, c = (f - 31) % 3;
    if constexpr (DIM == 3) {
      dv = pf_value<DIM, MIXED>(s, PF<3>::F, r * 3 + c, p);
    } else {
      dv = (r < 2 && c < 2) ? pf_value<DIM, MIXED>(s, PF<2>::F, r * 2 + c, p)
                            : (r == 2 && c == 2 ? 1.0 : 0.0);
    }
  } else if (f == 40) {  // initialise_mapping_matrix: no affine velocity update
    kind = 3;
  } else if (f < 50) {  // mapping matrix
    dv = 0.0;
  } else if (f == 50) {  // status
    kind = 3;
    uv = s.cell[p] >= 0 ? 1 : 0;
  } else if (f == 51) {  // cell id
    kind = 1;
    uv = (uint64_t)(int64_t)s.cell[p];
  } else if (f == 52) {
    kind = 2;
    uv = (uint32_t)a.material_id[s.mat[p]];
  } else if (f == 53) {
    kind = 2;
    uv = a.nstate[s.mat[p]];
  } else {  // svars[0..19]
    const int k = f - 54;
    dv = (k < SV_N && a.nstate[s.mat[p]] > 0) ? svar_value<DIM, MIXED>(s, k, p) : 0.0;
  }
}

template <int DIM, bool MIXED>
__global__ void __launch_bounds__(256) k_pod_pack(DevState s, PodAux a, PodLayout L,
                                                  const int32_t* list, int64_t count,
                                                  uint8_t* out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count * POD_NFIELDS) return;
  const int64_t i = t / POD_NFIELDS;
  const int f = (int)(t % POD_NFIELDS);
  const int64_t p = list[i];
  double dv;
  uint64_t uv;
  int kind;
  pod_field<DIM, MIXED>(s, a, f, p, dv, uv, kind);
  uint8_t* dst = out + i * L.record_size + L.offset[f];
  // sizes and alignments were checked on the host: 8-byte fields at 8-byte
  // offsets, 4-byte at 4-byte, records a multiple of 8 bytes
  if (kind == 0)
    *reinterpret_cast<double*>(dst) = dv;
  else if (kind == 1)
    *reinterpret_cast<uint64_t*>(dst) = uv;
  else if (kind == 2)
    *reinterpret_cast<uint32_t*>(dst) = (uint32_t)uv;
  else
    *dst = (uint8_t)(uv ? 1 : 0);
}

}  // namespace

namespace {

// F's storage in the device layout (2D: F00 F01 F10 F11; 3D: row-major 3 x 3)
// and the matching entries of the caller's row-major 3 x 3
template <int DIM>
__device__ __forceinline__ int f_row(int k) {
  return DIM == 2 ? (k < 2 ? k : k + 1) : k;
}
template <int DIM>
__device__ __forceinline__ bool f_diag(int k) {
  return DIM == 2 ? (k == 0 || k == 3) : (k % 4 == 0);
}
// strain Voigt entries kept in 2D: xx, yy, xy
__device__ __forceinline__ int e_row2(int k) { return k < 2 ? k : 3; }

template <int DIM, bool MIXED>
__global__ void __launch_bounds__(256) k_rows_to_state(DevState s, RowStage r, int any_mc) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ns = s.np;
  if (p >= ns) return;
  const bool live = p < r.n;
  auto row = [&](int64_t off, int w, int k) { return live ? r.base[off + p * w + k] : 0.; };
  constexpr int NS = PF<DIM>::NS, NE = PF<DIM>::NE, NFG = PF<DIM>::NFG;
  if constexpr (!MIXED) {
    double* pf = s.pf;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      pf[(PF<DIM>::X + d) * ns + p] = row(r.x, 3, d);
      pf[(PF<DIM>::U + d) * ns + p] = row(r.u, 3, d);
      pf[(PF<DIM>::V + d) * ns + p] = row(r.v, 3, d);
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) pf[(PF<DIM>::S + k) * ns + p] = row(r.stress, 6, k);
#pragma unroll
    for (int k = 0; k < NE; ++k)
      pf[(PF<DIM>::E + k) * ns + p] = row(r.strain, 6, DIM == 2 ? e_row2(k) : k);
#pragma unroll
    for (int k = 0; k < NFG; ++k) pf[(PF<DIM>::F + k) * ns + p] = row(r.F, 9, f_row<DIM>(k));
    pf[PF<DIM>::VOL * ns + p] = row(r.volume, 1, 0);
    pf[PF<DIM>::RHO * ns + p] = row(r.density, 1, 0);
    pf[PF<DIM>::MASS * ns + p] = row(r.mass, 1, 0);
    if (any_mc)
#pragma unroll
      for (int k = 0; k < SV_N; ++k) s.sv[(int64_t)k * ns + p] = row(r.svars, 9, k);
  } else {
    double* px = s.pf;
    float* pm = s.pm;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      px[(PDX<DIM>::X + d) * ns + p] = row(r.x, 3, d);
      px[(PDX<DIM>::U + d) * ns + p] = row(r.u, 3, d);
      pm[(PM<DIM>::V + d) * ns + p] = (float)row(r.v, 3, d);
    }
    px[PDX<DIM>::PDS * ns + p] = any_mc ? row(r.svars, 9, SV_PD) : 0.;
#pragma unroll
    for (int k = 0; k < NS; ++k) pm[(PM<DIM>::S + k) * ns + p] = (float)row(r.stress, 6, k);
#pragma unroll
    for (int k = 0; k < NE; ++k)
      pm[(PM<DIM>::E + k) * ns + p] = (float)row(r.strain, 6, DIM == 2 ? e_row2(k) : k);
#pragma unroll
    for (int k = 0; k < NFG; ++k)
      pm[(PM<DIM>::H + k) * ns + p] =
          (float)(row(r.F, 9, f_row<DIM>(k)) - (f_diag<DIM>(k) ? 1. : 0.));
    pm[PM<DIM>::V0 * ns + p] = (float)row(r.volume, 1, 0);
    pm[PM<DIM>::RHO0 * ns + p] = (float)row(r.density, 1, 0);
    pm[PM<DIM>::JP * ns + p] = 0.f;
    pm[PM<DIM>::MASS * ns + p] = (float)row(r.mass, 1, 0);
    if (any_mc)
#pragma unroll
      for (int k = 0; k < SVF_N; ++k) s.svf[(int64_t)k * ns + p] = (float)row(r.svars, 9, k);
  }
}

template <int DIM, bool MIXED>
__global__ void __launch_bounds__(256) k_state_to_rows(DevState s, RowStage r, int any_mc) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= r.n) return;
  const int64_t ns = s.np;
  double* b = r.base;
  auto put = [&](int64_t off, int w, int k, double v) {
    if (off >= 0) b[off + p * w + k] = v;
  };
  constexpr int NS = PF<DIM>::NS, NE = PF<DIM>::NE, NFG = PF<DIM>::NFG;
  // the device fields in FP64 (mixed: FP32 ones widened, as the host reads them)
  double x[DIM], u[DIM], v[DIM], sg[NS], ep[NE], F[NFG], vol, rho, mass, sv[SV_N];
  if constexpr (!MIXED) {
    const double* pf = s.pf;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      x[d] = pf[(PF<DIM>::X + d) * ns + p];
      u[d] = pf[(PF<DIM>::U + d) * ns + p];
      v[d] = pf[(PF<DIM>::V + d) * ns + p];
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) sg[k] = pf[(PF<DIM>::S + k) * ns + p];
#pragma unroll
    for (int k = 0; k < NE; ++k) ep[k] = pf[(PF<DIM>::E + k) * ns + p];
#pragma unroll
    for (int k = 0; k < NFG; ++k) F[k] = pf[(PF<DIM>::F + k) * ns + p];
    vol = pf[PF<DIM>::VOL * ns + p];
    rho = pf[PF<DIM>::RHO * ns + p];
    mass = pf[PF<DIM>::MASS * ns + p];
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = any_mc ? s.sv[(int64_t)k * ns + p] : 0.;
  } else {
    const double* px = s.pf;
    const float* pm = s.pm;
    auto m = [&](int f) { return (double)pm[(int64_t)f * ns + p]; };
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      x[d] = px[(PDX<DIM>::X + d) * ns + p];
      u[d] = px[(PDX<DIM>::U + d) * ns + p];
      v[d] = m(PM<DIM>::V + d);
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) sg[k] = m(PM<DIM>::S + k);
#pragma unroll
    for (int k = 0; k < NE; ++k) ep[k] = m(PM<DIM>::E + k);
#pragma unroll
    for (int k = 0; k < NFG; ++k) F[k] = m(PM<DIM>::H + k) + (f_diag<DIM>(k) ? 1. : 0.);
    const double jp = m(PM<DIM>::JP);
    vol = m(PM<DIM>::V0) * (1. + jp);
    rho = m(PM<DIM>::RHO0) / (1. + jp);
    mass = m(PM<DIM>::MASS);
#pragma unroll
    for (int k = 0; k < SV_N; ++k) sv[k] = 0.;
    if (any_mc) {
#pragma unroll
      for (int k = 0; k < SVF_N; ++k) sv[k] = (double)s.svf[(int64_t)k * ns + p];
      sv[SV_PD] = px[PDX<DIM>::PDS * ns + p];
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    put(r.x, 3, d, d < DIM ? x[d] : 0.);
    put(r.u, 3, d, d < DIM ? u[d] : 0.);
    put(r.v, 3, d, d < DIM ? v[d] : 0.);
  }
  if constexpr (DIM == 3) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      put(r.stress, 6, k, sg[k]);
      put(r.strain, 6, k, ep[k]);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) put(r.F, 9, k, F[k]);
  } else {
    const double s6[6] = {sg[0], sg[1], sg[2], sg[3], 0., 0.};
    const double e6[6] = {ep[0], ep[1], 0., ep[2], 0., 0.};
    const double f9[9] = {F[0], F[1], 0., F[2], F[3], 0., 0., 0., 1.};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      put(r.stress, 6, k, s6[k]);
      put(r.strain, 6, k, e6[k]);
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) put(r.F, 9, k, f9[k]);
  }
  put(r.volume, 1, 0, vol);
  put(r.density, 1, 0, rho);
  put(r.mass, 1, 0, mass);
#pragma unroll
  for (int k = 0; k < SV_N; ++k) put(r.svars, 9, k, sv[k]);
}

}  // namespace

void launch_rows_to_state(int dim, bool mixed, bool any_mc, const DevState& s, const RowStage& r,
                          cudaStream_t st) {
  const unsigned nb = (unsigned)((s.np + 255) / 256);
  if (nb == 0) return;
  if (dim == 2)
    mixed ? k_rows_to_state<2, true><<<nb, 256, 0, st>>>(s, r, any_mc)
          : k_rows_to_state<2, false><<<nb, 256, 0, st>>>(s, r, any_mc);
  else
    mixed ? k_rows_to_state<3, true><<<nb, 256, 0, st>>>(s, r, any_mc)
          : k_rows_to_state<3, false><<<nb, 256, 0, st>>>(s, r, any_mc);
}

void launch_state_to_rows(int dim, bool mixed, bool any_mc, const DevState& s, const RowStage& r,
                          cudaStream_t st) {
  const unsigned nb = (unsigned)((r.n + 255) / 256);
  if (nb == 0) return;
  if (dim == 2)
    mixed ? k_state_to_rows<2, true><<<nb, 256, 0, st>>>(s, r, any_mc)
          : k_state_to_rows<2, false><<<nb, 256, 0, st>>>(s, r, any_mc);
  else
    mixed ? k_state_to_rows<3, true><<<nb, 256, 0, st>>>(s, r, any_mc)
          : k_state_to_rows<3, false><<<nb, 256, 0, st>>>(s, r, any_mc);
}

void launch_pod_pack(int dim, bool mixed, const DevState& s, const PodAux& a, const PodLayout& L,
                     const int32_t* list, int64_t count, uint8_t* out, cudaStream_t st) {
  if (count <= 0) return;
  const int64_t threads = count * POD_NFIELDS;
  const unsigned blocks = (unsigned)((threads + 255) / 256);
  if (dim == 2) {
    if (mixed)
      k_pod_pack<2, true><<<blocks, 256, 0, st>>>(s, a, L, list, count, out);
    else
      k_pod_pack<2, false><<<blocks, 256, 0, st>>>(s, a, L, list, count, out);
  } else {
    if (mixed)
      k_pod_pack<3, true><<<blocks, 256, 0, st>>>(s, a, L, list, count, out);
    else
      k_pod_pack<3, false><<<blocks, 256, 0, st>>>(s, a, L, list, count, out);
  }
}

}  // namespace mpm_b200
