// Predictor / corrector update of one particle (time_int.cu:3-48 and
// :50-92), shared by the fused governing epilogue, the stand-alone
// integration kernels and the learned-correction epilogue.
#pragma once
#include "zsph_internal.cuh"

namespace zsph {

// Precision form: move offset o (cell coordinate c) into [0, gs) again after
// an update smaller than one cell; a cell outside the grid becomes kCellMask,
// which the next hash treats as out of the grid.
__device__ __forceinline__ void renormalize(float& o, int& c, float gs, int dim) {
  if (o >= gs) {
    o -= gs;
    c += 1;
  } else if (o < 0.0f) {
    o += gs;
    c -= 1;
  }
  if (c < 0 || c >= dim) c = kCellMask;
}

// time_int.cu:3-48 / :50-92 for one fluid particle, writing into `out`
// (which may alias `in`).  Non-fluid particles are copied unchanged.
// PRECISE (precision form, out != in): positions are cell offsets; the
// correction is x(n+1) = x(n+1/2) + v(n+1/2) dt - v(n) dt/2 (equal to
// time_int.cu:65-73 in exact arithmetic, and free of the old cell), and the
// cell of the result is written to kp.c3o.
template <int MODE, bool PRECISE = false>
__device__ __forceinline__ void integrate_one(const KParams& kp, const zsph_ptc_t& in, const zsph_ptc_t& out,
                                              int i, float4 acc) {
  const zsph_gpu_param_t& p = kp.p;
  const float3 pos = make_float3(in.pos[3 * i], in.pos[3 * i + 1], in.pos[3 * i + 2]);
  const float3 vel = make_float3(in.vel[3 * i], in.vel[3 * i + 1], in.vel[3 * i + 2]);
  const float2 rp = reinterpret_cast<const float2*>(in.rhop)[i];
  const int type = in.type[i];
  const bool alias = in.pos == out.pos;
  float3 tp = make_float3(in.tmp_pos[3 * i], in.tmp_pos[3 * i + 1], in.tmp_pos[3 * i + 2]);
  float3 tv = make_float3(in.tmp_vel[3 * i], in.tmp_vel[3 * i + 1], in.tmp_vel[3 * i + 2]);
  float2 trp = reinterpret_cast<const float2*>(in.tmp_rhop)[i];
  float3 np = pos, nv = vel;
  float2 nrp = rp;
  if (type == 1) {
    if (MODE == 1) {  // prediction
      tp = pos; tv = vel; trp = rp;
      np.x += vel.x * p.half_dt; np.y += vel.y * p.half_dt; np.z += vel.z * p.half_dt;
      nv.x += acc.x * p.half_dt; nv.y += acc.y * p.half_dt; nv.z += acc.z * p.half_dt;
      nrp.x += acc.w * p.half_dt;
    } else {  // correction
      if (PRECISE) {
        np.x = pos.x + (vel.x * p.half_dt * 2.0f - tv.x * p.half_dt);
        np.y = pos.y + (vel.y * p.half_dt * 2.0f - tv.y * p.half_dt);
        np.z = pos.z + (vel.z * p.half_dt * 2.0f - tv.z * p.half_dt);
      } else {
        np.x = tp.x + vel.x * p.half_dt * 2.0f;
        np.y = tp.y + vel.y * p.half_dt * 2.0f;
        np.z = tp.z + vel.z * p.half_dt * 2.0f;
      }
      nv.x = tv.x + acc.x * p.half_dt * 2.0f;
      nv.y = tv.y + acc.y * p.half_dt * 2.0f;
      nv.z = tv.z + acc.z * p.half_dt * 2.0f;
      nrp.x = trp.x + acc.w * p.half_dt * 2.0f;
    }
    if (nrp.x < p.rho0) nrp.x = p.rho0;
    nrp.y = p.cs2 * (nrp.x - p.rho0);
  } else if (alias) {
    return;
  }
  if (PRECISE) {
    int c = kp.c3n[i];
    if (type == 1) {
      int3 cc = unpack_cell(c);
      renormalize(np.x, cc.x, p.grid_size, p.grid_xdim);
      renormalize(np.y, cc.y, p.grid_size, p.grid_ydim);
      renormalize(np.z, cc.z, p.grid_size, p.grid_zdim);
      c = pack_cell(cc.x, cc.y, cc.z);
    }
    kp.c3o[i] = c;
  }
  out.pos[3 * i] = np.x; out.pos[3 * i + 1] = np.y; out.pos[3 * i + 2] = np.z;
  out.vel[3 * i] = nv.x; out.vel[3 * i + 1] = nv.y; out.vel[3 * i + 2] = nv.z;
  reinterpret_cast<float2*>(out.rhop)[i] = nrp;
  if (!alias || (MODE == 1 && type == 1)) {
    out.tmp_pos[3 * i] = tp.x; out.tmp_pos[3 * i + 1] = tp.y; out.tmp_pos[3 * i + 2] = tp.z;
    out.tmp_vel[3 * i] = tv.x; out.tmp_vel[3 * i + 1] = tv.y; out.tmp_vel[3 * i + 2] = tv.z;
    reinterpret_cast<float2*>(out.tmp_rhop)[i] = trp;
  }
  if (!alias) {
    out.type[i] = type;
    out.table[i] = in.table[i];
  }
}

}  // namespace zsph
