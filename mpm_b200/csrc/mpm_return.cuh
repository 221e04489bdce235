// mpm_return.cuh -- the MohrCoulomb plastic return as a loop of uniform passes.
//
// MohrCoulomb<Tdim>::compute_stress (mohr_coulomb.tcc:348-513) evaluates the
// stress invariants and yield state of a stress, and mostly dF/dsigma and
// dP/dsigma of it, at the trial stress, at the old stress, after every
// correction and at the final stress.  Written as straight-line code, as in
// mc_stress, each of these evaluations is a separate copy of the same three
// heavy pieces: inlined, the dense return kernels outgrow the instruction
// cache; called out of line, every call passes its arrays through the stack.
// Here the return is one loop whose every pass evaluates, at a single site,
// the invariants and yield state of the point's current stress and, where its
// phase needs them, dF/dsigma and dP/dsigma -- then makes the phase's small
// update.  Each heavy piece is inlined once, everything can stay in
// registers, and the lanes of a warp that are in different phases run the
// same pass code together.  Per point the evaluations, their inputs and their
// order are those of mc_stress<R, PD, false>, so the results are the same.
#pragma once

#include "mpm_math.cuh"

namespace mpm_b200 {

enum { MR_TRIAL = 0, MR_OLD, MR_TRIAL_DF, MR_LOOP, MR_FINAL };

// One point's return in progress.
template <typename R>
struct McPoint {
  int phase, itr, yt_trial;
  R trial[6], upd[6], sv[SV_N];
  R pd;   // plastic deviatoric strain at the start of the update
  R dpd;  // its increment
  R yield_trial;
  LodeTrig<R> lt;
  FrictionTrig<R> ft;
};

// The part of mc_stress before its first invariants: softening of the state,
// elastic predictor, separated state.  q.sv, with the plastic deviatoric strain
// in SV_PD, is loaded by the caller.  True when the point is finished here
// (separated: out = 0 and q.sv final).
template <typename R>
__device__ __forceinline__ bool mc_begin(const MaterialT<R>& m, const R* stress, const R* dstrain,
                                         R density, McPoint<R>& q, R* out) {
  q.pd = q.sv[SV_PD];
  const R pdstrain = q.pd;
  if (m.softening && pdstrain > m.pd_peak) {
    if (pdstrain < m.pd_res) {
      q.sv[SV_PHI] = m.phi_res + ((m.phi_peak - m.phi_res) * (pdstrain - m.pd_res) /
                                  (m.pd_peak - m.pd_res));
      q.sv[SV_PSI] = m.psi_res + ((m.psi_peak - m.psi_res) * (pdstrain - m.pd_res) /
                                  (m.pd_peak - m.pd_res));
      q.sv[SV_COH] = m.c_res + ((m.c_peak - m.c_res) * (pdstrain - m.pd_res) / (m.pd_peak - m.pd_res));
    } else {
      q.sv[SV_PHI] = m.phi_res;
      q.sv[SV_PSI] = m.psi_res;
      q.sv[SV_COH] = m.c_res;
    }
    const R apex = q.sv[SV_COH] / tan(q.sv[SV_PHI]);
    if (q.sv[SV_TC] > apex) q.sv[SV_TC] = check_low(apex);
  }
  q.sv[SV_YIELD] = R(0);
  {
    R t[6];
    de_mul(m, dstrain, t);
#pragma unroll
    for (int i = 0; i < 6; ++i) q.trial[i] = stress[i] + t[i];
  }
  if (density <= m.min_packing * m.grain_density) {
    q.sv[SV_PD] = q.pd + sqrt(R(3) * mu_j2(q.trial)) / R(3) / m.shear;
    q.sv[SV_YIELD] = R(3);
#pragma unroll
    for (int i = 0; i < 6; ++i) out[i] = R(0);
    return true;
  }
  q.ft = friction_trig(m, q.sv);
  q.phase = MR_TRIAL;
  q.itr = 0;
  q.yt_trial = MC_ELASTIC;
  q.dpd = R(0);
  q.yield_trial = R(0);
  return false;
}

// One pass: the invariants and yield state of the point's current stress X
// (trial, old, trial again, corrected), dF/dsigma and dP/dsigma of X where the
// phase needs them, then the phase's update.  True when the point is
// finished (out and q.sv final).
//
// The trial stress's dF/dsigma is needed only when the old stress is off the
// yield surface; mc_stress keeps the trial invariants for it, here the pass
// MR_TRIAL_DF evaluates them again (the same inputs give the same values)
// into q.sv, which changes only epsilon, rho and theta there -- evaluated again
// at the corrected stress before anything else reads them.
template <typename R>
__device__ __forceinline__ bool mc_pass(const MaterialT<R>& m, const R* stress, const R* dstrain,
                                        McPoint<R>& q, R* out) {
  const R Tolerance = R(1E-1);
  const int ph = q.phase;
  R X[6];
#pragma unroll
  for (int i = 0; i < 6; ++i)
    X[i] = (ph == MR_TRIAL || ph == MR_TRIAL_DF) ? q.trial[i] : (ph == MR_OLD ? stress[i] : q.upd[i]);
  mc_invariants(X, q.sv, q.lt);
  R yf[2];
  const int yt = mc_yield_state(yf, q.sv, q.lt, q.ft);
  const bool converged = yf[0] < Tolerance && yf[1] < Tolerance;
  R softening = R(0), dp_dq = R(0), df[6], dp[6];
  if (ph == MR_OLD || ph == MR_TRIAL_DF || (ph == MR_LOOP && !converged))
    mc_df_dp(m, ph == MR_TRIAL_DF ? q.yt_trial : yt, q.sv, q.lt, q.ft, q.pd, X, df, dp, &dp_dq,
             &softening);
  if (ph == MR_TRIAL) {
    if (yt == MC_ELASTIC) {
      q.sv[SV_YIELD] = R(0);
#pragma unroll
      for (int i = 0; i < 6; ++i) out[i] = q.trial[i];
      return true;
    }
    q.yt_trial = yt;
    if (yt == MC_TENSILE) {
      q.sv[SV_YIELD] = R(2);
      q.yield_trial = yf[0];
    }
    if (yt == MC_SHEAR) {
      q.sv[SV_YIELD] = R(1);
      q.yield_trial = yf[1];
    }
    q.phase = MR_OLD;
    return false;
  }
  if (ph == MR_OLD) {
    R yield = huge_value<R>();
    if (yt == MC_TENSILE) yield = yf[0];
    if (yt == MC_SHEAR) yield = yf[1];
    if (fabs(yield) < Tolerance) {
      const R lambda = row_de_dot(m, df, dstrain) / (row_de_dot(m, df, dp) + softening);
#pragma unroll
      for (int i = 0; i < 6; ++i) q.upd[i] = q.trial[i];
      sub_lambda_de(m, lambda, dp, q.upd);
      q.dpd = lambda * dp_dq;
      q.phase = MR_LOOP;
    } else {
      q.phase = MR_TRIAL_DF;
    }
    return false;
  }
  if (ph == MR_TRIAL_DF) {
    const R lambda_trial = q.yield_trial / (row_de_dot(m, df, dp) + softening);
#pragma unroll
    for (int i = 0; i < 6; ++i) q.upd[i] = q.trial[i];
    sub_lambda_de(m, lambda_trial, dp, q.upd);
    q.dpd = lambda_trial * dp_dq;
    q.phase = MR_LOOP;
    return false;
  }
  if (ph == MR_LOOP && !converged) {
    if (yt == MC_TENSILE) q.yield_trial = yf[0];
    if (yt == MC_SHEAR) q.yield_trial = yf[1];
    const R lambda_trial = q.yield_trial / (row_de_dot(m, df, dp) + softening);
    sub_lambda_de(m, lambda_trial, dp, q.upd);
    q.dpd += lambda_trial * dp_dq;
    if (++q.itr == 100) q.phase = MR_FINAL;
    return false;
  }
  // converged (the invariants of the final stress are in q.sv), or MR_FINAL
  // after the 100th correction (they were just evaluated)
  q.sv[SV_PD] = q.pd + q.dpd;
#pragma unroll
  for (int i = 0; i < 6; ++i) out[i] = q.upd[i];
  return true;
}

// The full MohrCoulomb update of mc_compute_stress<R, R> as passes: sv holds
// the state variables with the plastic deviatoric strain in SV_PD (updated in
// place), corrections receives the number of return corrections.
template <typename R>
__device__ __forceinline__ void mc_return(const MaterialT<R>& m, const R* stress, const R* dstrain,
                                          R density, R* sv, R* out, int* corrections) {
  McPoint<R> q;
#pragma unroll
  for (int k = 0; k < SV_N; ++k) q.sv[k] = sv[k];
  if (!mc_begin(m, stress, dstrain, density, q, out)) {
    while (!mc_pass(m, stress, dstrain, q, out)) {
    }
  }
#pragma unroll
  for (int k = 0; k < SV_N; ++k) sv[k] = q.sv[k];
  *corrections = q.itr;
}

}  // namespace mpm_b200
