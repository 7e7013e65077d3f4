// fk_jac.cu — fused forward kinematics + frame Jacobians for sm_100a.
//
// Work mapping: one warp owns one configuration at a time (persistent grid,
// warps stride over the batch).  Inside the warp:
//   * lanes load q coalesced into shared memory;
//   * lane j builds liMi_j = placement_j * T_j(q_j) for its joint(s)
//     (forward.py:110-123 evaluates the same product joint by joint);
//   * world placements oMi come from pointer jumping over the parent table:
//     T_j <- T_anc(j) * T_j, anc(j) <- anc(anc(j)), ceil(log2 depth) rounds, so a
//     tree of depth d costs log2(d) composes per lane instead of a serial walk
//     (forward.py:125-129);
//   * target (frame) placements oMf = oMi[parent] * placement (forward.py:213-216);
//   * Jacobian columns are generated directly from the column's world axis a and
//     origin o (rotation: [a x (p_f - o); a] in LOCAL_WORLD_ALIGNED, [o x a; a] in
//     WORLD; translation: [a; 0]), zero outside the target's support — the
//     O(nj * 6 * nv) per-joint parent copies of jacobian.py:45-79 never happen;
//   * every output block of the configuration (J: n_targets*6*nv floats,
//     poses: n*7 floats) is assembled in shared memory and written with one
//     cp.async.bulk store (TMA bulk copy, full 128-B lines), so HBM sees only
//     the algorithmic bytes.  A J block above 16 KB (all 32 joints of a humanoid:
//     27.6 KB) goes out in pieces of a few targets through two alternating
//     buffers, so that its size does not cap the warps per SM;
//   * in from-poses mode (compute_joint_jacobians) the next configuration's
//     placements are loaded into registers while the current one is written.
#include <cuda_runtime.h>
#include <stdint.h>

#include "br_common.cuh"
#include "br_lie.cuh"
#include "br_fk.cuh"

namespace br {

enum : uint32_t { OUT_OMI = 1u, OUT_LIMI = 2u, OUT_TPOSE = 4u, OUT_JAC = 8u };

struct FkParams {
  const float* q;        // [B, nq]           (from-q mode)
  const float* oMi_in;   // [B, nj, 7]        (from-poses mode)
  int64_t batch;
  float* oMi;            // [B, nj, 7]        or null
  float* liMi;           // [B, nj, 7]        or null
  float* tpose;          // [B, nt, 7]        or null
  float* jac;            // [B, nt, 6, nv]    or null
  int32_t nt;
  uint32_t outputs;      // OUT_* bits
  uint32_t bulk;         // OUT_* bits whose blocks are 16-byte aligned -> TMA bulk store
  int32_t chunk;         // targets per staged piece of the J block (>= nt: the whole block)
  int32_t targets[BR_MAX_TARGETS];
};

// Shared-memory layout (in floats; every region starts on a 16-byte boundary).
struct Layout {
  // CTA-wide tables
  int parent, jtype, idxq, axis, place, cjoint, ckind, caxis, tparent, tplace, tmask, pairoff, pairs, npairs;
  int cta_floats;
  // per-warp regions
  int q, poseT, poseQ, anc, colA, colO, tgt, sJ, sT, sOMi, sLiMi;
  int warp_floats;
  // chunk: targets per staged piece of a configuration's J block.  chunk >= nt stages the
  // whole block in one buffer; a smaller (even) chunk stages it piece by piece in two
  // alternating buffers, so a large block (all joints of a humanoid: 27.6 KB) does not
  // limit the warps per SM.
  __host__ __device__ Layout(int nj, int nq, int nv, int nt, uint32_t outputs, int chunk) {
    int o = 0;
    parent = o; o += round4(nj);
    jtype = o; o += round4(nj);
    idxq = o; o += round4(nj);
    axis = o; o += 4 * nj;
    place = o; o += 8 * nj;
    cjoint = o; o += round4(nv);
    ckind = o; o += round4(nv);
    caxis = o; o += 4 * nv;
    tparent = o; o += round4(nt);
    tplace = o; o += 8 * nt;
    tmask = o; o += round4(2 * nt);                              // uint64 column mask per target
    pairoff = o; o += round4(nt);
    pairs = o; o += (outputs & OUT_JAC) ? round4(nt * nv) : 0;   // (target << 8 | column) with support
    npairs = o; o += 4;
    cta_floats = o;
    o = 0;
    q = o; o += round4(nq);
    poseT = o; o += 4 * nj;                                      // world translation (x, y, z, 0)
    poseQ = o; o += 4 * nj;                                      // world quaternion
    anc = o; o += round4(nj);
    colA = o; o += 4 * nv;                                       // world column axis
    colO = o; o += 4 * nv;                                       // world column origin
    tgt = o; o += 8 * nt;
    sJ = o; o += (outputs & OUT_JAC) ? (chunk < nt ? 2 * round4(chunk * 6 * nv) : round4(nt * 6 * nv)) : 0;
    sT = o; o += (outputs & OUT_TPOSE) ? round4(nt * 7) : 0;
    sOMi = o; o += (outputs & OUT_OMI) ? round4(nj * 7) : 0;
    sLiMi = o; o += (outputs & OUT_LIMI) ? round4(nj * 7) : 0;
    warp_floats = o;
  }
};

template <int kRef, bool kFromQ>
__global__ void fk_jac_kernel(const br_tree_t tree, const FkParams p) {
  extern __shared__ __align__(16) float smem[];
  const int nj = tree.njoints, nq = tree.nq, nv = tree.nv, nt = p.nt;
  const bool want_jac = (p.outputs & OUT_JAC) != 0;
  const Layout L(nj, nq, nv, nt, p.outputs, p.chunk);
  const bool chunked = want_jac && p.chunk < nt;
  float* cta = smem;
  int* s_parent = reinterpret_cast<int*>(cta + L.parent);
  int* s_jtype = reinterpret_cast<int*>(cta + L.jtype);
  int* s_idxq = reinterpret_cast<int*>(cta + L.idxq);
  float* s_axis = cta + L.axis;
  float* s_place = cta + L.place;
  int* s_cjoint = reinterpret_cast<int*>(cta + L.cjoint);
  int* s_ckind = reinterpret_cast<int*>(cta + L.ckind);
  float* s_caxis = cta + L.caxis;
  int* s_tparent = reinterpret_cast<int*>(cta + L.tparent);
  float* s_tplace = cta + L.tplace;
  unsigned long long* s_tmask = reinterpret_cast<unsigned long long*>(cta + L.tmask);
  int* s_pairoff = reinterpret_cast<int*>(cta + L.pairoff);
  int* s_pairs = reinterpret_cast<int*>(cta + L.pairs);
  int* s_npairs = reinterpret_cast<int*>(cta + L.npairs);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpc = blockDim.x >> 5;

  for (int i = threadIdx.x; i < nj; i += blockDim.x) {
    s_parent[i] = tree.parent[i];
    s_jtype[i] = tree.jtype[i];
    s_idxq[i] = tree.idx_q[i];
    for (int k = 0; k < 4; ++k) s_axis[4 * i + k] = tree.axis[4 * i + k];
    for (int k = 0; k < 8; ++k) s_place[8 * i + k] = tree.placement[8 * i + k];
  }
  for (int c = threadIdx.x; c < nv; c += blockDim.x) {
    s_cjoint[c] = tree.col_joint[c];
    s_ckind[c] = tree.col_kind[c];
    for (int k = 0; k < 4; ++k) s_caxis[4 * c + k] = tree.col_axis[4 * c + k];
  }
  for (int s = threadIdx.x; s < nt; s += blockDim.x) {
    const int id = p.targets[s];
    int par;
    if (id >= 0) {
      par = tree.frame_parent[id];
      for (int k = 0; k < 8; ++k) s_tplace[8 * s + k] = tree.frame_placement[8 * id + k];
    } else {
      par = -id - 1;
      for (int k = 0; k < 8; ++k) s_tplace[8 * s + k] = (k == 7) ? 1.f : 0.f;  // identity
    }
    s_tparent[s] = par;
  }
  __syncthreads();
  // Columns with a non-zero Jacobian entry for each target: col_joint[c] supports the
  // target's parent joint.  The list of such (target, column) pairs is the only part of
  // the J block that depends on q; the rest is zero and is written once below.
  for (int s = warp; s < nt; s += wpc) {
    const unsigned long long sup = tree.support[s_tparent[s]];
    unsigned long long m = 0ull;
    for (int c0 = 0; c0 < nv; c0 += kWarp) {
      const int c = c0 + lane;
      const bool in = c < nv && ((sup >> s_cjoint[c]) & 1ull);
      m |= (unsigned long long)__ballot_sync(0xffffffffu, in) << c0;
    }
    if (lane == 0) s_tmask[s] = m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int off = 0;
    for (int s = 0; s < nt; ++s) {
      s_pairoff[s] = off;
      off += __popcll(s_tmask[s]);
    }
    s_npairs[0] = off;
  }
  __syncthreads();
  if (want_jac) {
    for (int s = warp; s < nt; s += wpc) {
      const unsigned long long m = s_tmask[s];
      for (int c = lane; c < nv; c += kWarp)
        if ((m >> c) & 1ull) s_pairs[s_pairoff[s] + __popcll(m & ((1ull << c) - 1ull))] = (s << 8) | c;
    }
  }
  const int npairs = s_npairs[0];

  float* w = smem + L.cta_floats + warp * L.warp_floats;
  float* wq = w + L.q;
  float* wpT = w + L.poseT;
  float* wpQ = w + L.poseQ;
  int* wanc = reinterpret_cast<int*>(w + L.anc);
  float* wcA = w + L.colA;
  float* wcO = w + L.colO;
  float* wtgt = w + L.tgt;
  float* sJ = w + L.sJ;
  float* sT = w + L.sT;
  float* sOMi = w + L.sOMi;
  float* sLiMi = w + L.sLiMi;
  const int cfl = chunked ? round4(p.chunk * 6 * nv) : 0;  // floats per chunk buffer
  if (want_jac && !chunked) {  // the chunked staging buffers are cleared before each piece
    const int n = round4(nt * 6 * nv) / 4;
    for (int i = lane; i < n; i += kWarp) reinterpret_cast<float4*>(sJ)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();
  const int rounds = tree.rounds;
  const int64_t stride = (int64_t)gridDim.x * wpc;

  // q of the warp's next configuration is loaded into registers one iteration
  // ahead, so its global-load latency overlaps the current configuration's work
  // (nq <= BR_MAX_NQ = 128: at most 4 values per lane)
  float qn[4];
  const int64_t b0 = (int64_t)blockIdx.x * wpc + warp;
  if (kFromQ && b0 < p.batch) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = lane + kWarp * k;
      qn[k] = i < nq ? __ldg(p.q + b0 * nq + i) : 0.f;
    }
  }
  // likewise the next configuration's joint placements in from-poses mode
  // (nj * 7 <= BR_MAX_JOINTS * 7 = 448 floats: at most 14 values per lane)
  constexpr int kPoseRegs = (BR_MAX_JOINTS * 7 + kWarp - 1) / kWarp;
  float on[kPoseRegs];
  if (!kFromQ && b0 < p.batch) {
#pragma unroll
    for (int k = 0; k < kPoseRegs; ++k) {
      const int i = lane + kWarp * k;
      on[k] = i < nj * 7 ? __ldg(p.oMi_in + b0 * nj * 7 + i) : 0.f;
    }
  }
  uint32_t gc = 0;  // staged J pieces so far: piece gc uses buffer gc & 1
  for (int64_t b = b0; b < p.batch; b += stride) {
    // ---- world joint placements --------------------------------------
    if (kFromQ) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = lane + kWarp * k;
        if (i < nq) wq[i] = qn[k];
      }
      const int64_t bn = b + stride;
      if (bn < p.batch) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int i = lane + kWarp * k;
          qn[k] = i < nq ? __ldg(p.q + bn * nq + i) : 0.f;
        }
      }
      __syncwarp();
      Pose T[2];
      int anc[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int j = lane + kWarp * k;
        if (j < nj) {
          T[k] = local_transform(s_jtype[j], load_pose8(s_place + 8 * j), s_axis + 4 * j, wq + s_idxq[j]);
          anc[k] = s_parent[j];
        }
      }
      if (lane == 0) bulk_wait_read_all();  // staging buffers are free again
      __syncwarp();
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int j = lane + kWarp * k;
        if (j < nj) {
          store_split(wpT, wpQ, j, T[k]);
          wanc[j] = anc[k];
          if (p.outputs & OUT_LIMI) store_pose7(sLiMi + 7 * j, T[k]);
        }
      }
      __syncwarp();
      for (int r = 0; r < rounds; ++r) {
        Pose A[2];
        int aa[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int j = lane + kWarp * k;
          if (j < nj && anc[k] >= 0) {
            A[k] = load_split(wpT, wpQ, anc[k]);
            aa[k] = wanc[anc[k]];
          }
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int j = lane + kWarp * k;
          if (j < nj && anc[k] >= 0) {
            T[k] = compose(A[k], T[k]);
            anc[k] = aa[k];
            store_split(wpT, wpQ, j, T[k]);
            wanc[j] = anc[k];
          }
        }
        __syncwarp();
      }
      if (p.outputs & OUT_OMI) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int j = lane + kWarp * k;
          if (j < nj) store_pose7(sOMi + 7 * j, T[k]);
        }
      }
    } else {
      if (!chunked && lane == 0) bulk_wait_read_all();  // the whole-block buffer is free again
#pragma unroll
      for (int k = 0; k < kPoseRegs; ++k) {
        const int i = lane + kWarp * k;
        if (i < nj * 7) {
          const int j = i / 7, c = i - 7 * j;
          if (c < 3) wpT[4 * j + c] = on[k];
          else wpQ[4 * j + c - 3] = on[k];
        }
      }
      const int64_t bn = b + stride;
      if (bn < p.batch) {
#pragma unroll
        for (int k = 0; k < kPoseRegs; ++k) {
          const int i = lane + kWarp * k;
          on[k] = i < nj * 7 ? __ldg(p.oMi_in + bn * nj * 7 + i) : 0.f;
        }
      }
      __syncwarp();
    }

    // ---- target placements and world Jacobian columns --------------------
    for (int s = lane; s < nt; s += kWarp) {
      const Pose Tt = compose(load_split(wpT, wpQ, s_tparent[s]), load_pose8(s_tplace + 8 * s));
      store_pose8(wtgt + 8 * s, Tt);
      if (p.outputs & OUT_TPOSE) store_pose7(sT + 7 * s, Tt);
    }
    if (want_jac) {
      for (int c = lane; c < nv; c += kWarp) {
        const Pose Tj = load_split(wpT, wpQ, s_cjoint[c]);
        const float3 a = qrot(Tj.q, f3(s_caxis[4 * c], s_caxis[4 * c + 1], s_caxis[4 * c + 2]));
        *reinterpret_cast<float4*>(wcA + 4 * c) = make_float4(a.x, a.y, a.z, 0.f);
        *reinterpret_cast<float4*>(wcO + 4 * c) = make_float4(Tj.t.x, Tj.t.y, Tj.t.z, 0.f);
      }
    }
    __syncwarp();

    // the six entries of J column c for target s, rows nv floats apart from dst
    auto jac_pair = [&](int s, int c, float* dst) {
      const float4 a4 = *reinterpret_cast<const float4*>(wcA + 4 * c);
      const float3 a = f3(a4.x, a4.y, a4.z);
      float3 lin, ang;
      if (s_ckind[c] == 0) {
        const float4 o4 = *reinterpret_cast<const float4*>(wcO + 4 * c);
        const float3 o = f3(o4.x, o4.y, o4.z);
        if (kRef == BR_REF_WORLD) {
          lin = cross(o, a);                                   // hat(p_j) R S_ang  (jacobian.py:290-296)
        } else {
          const float4 pt = *reinterpret_cast<const float4*>(wtgt + 8 * s);
          lin = cross(a, sub(f3(pt.x, pt.y, pt.z), o));        // J_lin - hat(p_f) J_ang (jacobian.py:213-215)
        }
        ang = a;
      } else {
        lin = a;
        ang = f3(0.f, 0.f, 0.f);
      }
      if (kRef == BR_REF_LOCAL) {                              // R_f^T rows (jacobian.py:219-225)
        const float4 qt = *reinterpret_cast<const float4*>(wtgt + 8 * s + 4);
        lin = qrot_inv(qt, lin);
        ang = qrot_inv(qt, ang);
      }
      dst[0] = lin.x; dst[nv] = lin.y; dst[2 * nv] = lin.z;
      dst[3 * nv] = ang.x; dst[4 * nv] = ang.y; dst[5 * nv] = ang.z;
    };
    if (want_jac && !chunked) {
      for (int idx = lane; idx < npairs; idx += kWarp) {
        const int pr = s_pairs[idx];
        const int s = pr >> 8, c = pr & 255;
        jac_pair(s, c, sJ + s * 6 * nv + c);
      }
    }
    if (chunked) {
      // targets [t0, t1) at a time: clear a buffer, fill the piece's (target, column) pairs,
      // store it; the other buffer's store is still reading while this one is filled
      const bool bulkJ = (p.bulk & OUT_JAC) != 0;
      float* gJ = p.jac + b * (int64_t)nt * 6 * nv;
      for (int t0 = 0; t0 < nt; t0 += p.chunk) {
        const int t1 = t0 + p.chunk < nt ? t0 + p.chunk : nt;
        float* buf = sJ + (int)(gc & 1u) * cfl;
        ++gc;
        if (bulkJ && lane == 0) bulk_wait_read<1>();         // the store two pieces back has read buf
        __syncwarp();
        for (int i = lane; i < cfl / 4; i += kWarp) reinterpret_cast<float4*>(buf)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
        const int e1 = t1 < nt ? s_pairoff[t1] : npairs;
        for (int idx = s_pairoff[t0] + lane; idx < e1; idx += kWarp) {
          const int pr = s_pairs[idx];
          const int s = pr >> 8, c = pr & 255;
          jac_pair(s, c, buf + (s - t0) * 6 * nv + c);
        }
        const int n = (t1 - t0) * 6 * nv;
        if (bulkJ) {
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) {
            bulk_store(gJ + (int64_t)t0 * 6 * nv, buf, (uint32_t)n * 4u);
            bulk_commit();
          }
        } else {
          __syncwarp();
          warp_copy(gJ + (int64_t)t0 * 6 * nv, buf, n, lane);
        }
        __syncwarp();
      }
    }

    // ---- write the configuration's output blocks -----------------------
    fence_proxy_async_smem();
    __syncwarp();
    struct Out { uint32_t bit; float* g; const float* s; int n; };
    const Out outs[4] = {
        {OUT_JAC, p.jac ? p.jac + b * (int64_t)nt * 6 * nv : nullptr, sJ, nt * 6 * nv},
        {OUT_TPOSE, p.tpose ? p.tpose + b * (int64_t)nt * 7 : nullptr, sT, nt * 7},
        {OUT_OMI, p.oMi ? p.oMi + b * (int64_t)nj * 7 : nullptr, sOMi, nj * 7},
        {OUT_LIMI, p.liMi ? p.liMi + b * (int64_t)nj * 7 : nullptr, sLiMi, nj * 7}};
    bool issued = false;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
      if (!(p.outputs & outs[o].bit) || outs[o].n == 0 || (chunked && outs[o].bit == OUT_JAC)) continue;
      if (p.bulk & outs[o].bit) {
        if (lane == 0) bulk_store(outs[o].g, outs[o].s, (uint32_t)outs[o].n * 4u);
        issued = true;
      } else {
        warp_copy(outs[o].g, outs[o].s, outs[o].n, lane);
      }
    }
    if (issued && lane == 0) bulk_commit();
    __syncwarp();
  }
  if (lane == 0) bulk_wait_all();
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
const DeviceInfo& device_info() {
  static DeviceInfo info[16];
  int dev = 0;
  cudaGetDevice(&dev);
  DeviceInfo& d = info[dev & 15];
  if (d.device != dev) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    d.sms = prop.multiProcessorCount;
    d.max_smem_optin = (int)prop.sharedMemPerBlockOptin;
    d.l2_bytes = prop.l2CacheSize;
    d.device = dev;
  }
  return d;
}

int validate_tree(const br_tree_t* t) {
  if (!t) return BR_EINVAL;
  if (t->njoints < 1 || t->nq < 0 || t->nv < 0 || t->nframes < 0 || t->rounds < 0) return BR_EINVAL;
  if (t->njoints > BR_MAX_JOINTS || t->nv > BR_MAX_NV || t->nq > BR_MAX_NQ) return BR_ETOOBIG;
  if (!t->parent || !t->jtype || !t->idx_q || !t->idx_v || !t->axis || !t->placement || !t->support) return BR_EINVAL;
  if (t->nv > 0 && (!t->col_joint || !t->col_kind || !t->col_axis)) return BR_EINVAL;
  if (t->nframes > 0 && (!t->frame_parent || !t->frame_placement)) return BR_EINVAL;
  return BR_OK;
}

static int g_warps_per_cta = 8;

// A configuration's J block above kWholeBlockBytes is staged in pieces of about
// kPieceBytes (an even number of targets, so that every piece starts and ends on a
// 16-byte boundary of a 16-byte aligned block).  Measured on all 32 joint Jacobians of the
// humanoid at B = 16,384: pieces of 2 / 4 / 8 / 14 / 18 targets (2-16 KB) took 92 / 92 / 84 /
// 92 / 108 us; the 8 KB pieces leave one 8-warp CTA per SM and fewer, larger bulk copies.
constexpr int kWholeBlockBytes = 16384, kPieceBytes = 8192;

template <int kRef, bool kFromQ>
static int launch_fk(const br_tree_t& tree, FkParams p, cudaStream_t stream) {
  if (p.batch == 0) return BR_OK;
  p.chunk = p.nt;
  const int64_t jbytes = (int64_t)p.nt * 6 * tree.nv * 4;
  if ((p.outputs & OUT_JAC) && tree.nv > 0 && jbytes > kWholeBlockBytes) {
    int ch = (kPieceBytes / (6 * tree.nv * 4)) & ~1;
    p.chunk = ch < 2 ? 2 : ch;
  }
  const Layout L(tree.njoints, tree.nq, tree.nv, p.nt, p.outputs, p.chunk);
  const DeviceInfo& dev = device_info();
  int wpc = g_warps_per_cta;
  size_t bytes = 0;
  for (;;) {
    bytes = (size_t)(L.cta_floats + wpc * L.warp_floats) * sizeof(float);
    if ((int)bytes <= dev.max_smem_optin || wpc == 1) break;
    wpc >>= 1;
  }
  if ((int)bytes > dev.max_smem_optin) return BR_ETOOBIG;
  auto kern = fk_jac_kernel<kRef, kFromQ>;
  static int configured_bytes[16] = {0};
  int devslot = dev.device & 15;
  if ((int)bytes > configured_bytes[devslot]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    configured_bytes[devslot] = (int)bytes;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, wpc * kWarp, bytes);
  if (per_sm < 1) per_sm = 1;
  const int64_t need = (p.batch + wpc - 1) / wpc;
  const int64_t cap = (int64_t)per_sm * dev.sms;
  const int grid = (int)(need < cap ? need : cap);
  kern<<<grid, wpc * kWarp, bytes, stream>>>(tree, p);
  return (int)cudaGetLastError();
}

template <bool kFromQ>
static int dispatch_fk(const br_tree_t& tree, const FkParams& p, int32_t reference, cudaStream_t s) {
  switch (reference) {
    case BR_REF_WORLD: return launch_fk<BR_REF_WORLD, kFromQ>(tree, p, s);
    case BR_REF_LOCAL_WORLD_ALIGNED: return launch_fk<BR_REF_LOCAL_WORLD_ALIGNED, kFromQ>(tree, p, s);
    case BR_REF_LOCAL: return launch_fk<BR_REF_LOCAL, kFromQ>(tree, p, s);
    default: return BR_EINVAL;
  }
}

static int fill_targets(const br_tree_t* tree, FkParams& p, const int32_t* targets, int32_t n) {
  if (n < 0) return BR_EINVAL;
  if (n > BR_MAX_TARGETS) return BR_ETOOBIG;
  if (n > 0 && !targets) return BR_EINVAL;
  for (int i = 0; i < n; ++i) {
    const int id = targets[i];
    if (id >= 0 ? id >= tree->nframes : (-id - 1) >= tree->njoints) return BR_EINVAL;
    p.targets[i] = id;
  }
  p.nt = n;
  return BR_OK;
}

static uint32_t bulk_bit(uint32_t bit, const float* base, int64_t floats_per_item) {
  return (base && aligned16(base) && ((floats_per_item * 4) % 16) == 0) ? bit : 0u;
}

}  // namespace br

using namespace br;

extern "C" int br_forward_kinematics(const br_tree_t* tree, const float* q, int64_t batch,
                                     float* joint_pose_world, float* joint_pose_local,
                                     const int32_t* frame_ids, int32_t n_frames, float* frame_pose_world,
                                     void* stream) {
  int st = validate_tree(tree);
  if (st) return st;
  if (batch < 0 || (batch > 0 && tree->nq > 0 && !q)) return BR_EINVAL;
  if ((q && !aligned4(q))) return BR_EALIGN;
  FkParams p = {};
  p.q = q;
  p.batch = batch;
  p.oMi = joint_pose_world;
  p.liMi = joint_pose_local;
  p.tpose = frame_pose_world;
  st = fill_targets(tree, p, frame_ids, frame_pose_world ? n_frames : 0);
  if (st) return st;
  if ((joint_pose_world && !aligned4(joint_pose_world)) || (joint_pose_local && !aligned4(joint_pose_local)) ||
      (frame_pose_world && !aligned4(frame_pose_world)))
    return BR_EALIGN;
  p.outputs = (joint_pose_world ? OUT_OMI : 0u) | (joint_pose_local ? OUT_LIMI : 0u) |
              (frame_pose_world && p.nt > 0 ? OUT_TPOSE : 0u);
  p.bulk = bulk_bit(OUT_OMI, joint_pose_world, (int64_t)tree->njoints * 7) |
           bulk_bit(OUT_LIMI, joint_pose_local, (int64_t)tree->njoints * 7) |
           bulk_bit(OUT_TPOSE, frame_pose_world, (int64_t)p.nt * 7);
  if (!p.outputs) return BR_OK;
  return dispatch_fk<true>(*tree, p, BR_REF_LOCAL_WORLD_ALIGNED, (cudaStream_t)stream);
}

extern "C" int br_frame_jacobians(const br_tree_t* tree, const float* q, int64_t batch, const int32_t* targets,
                                  int32_t n_targets, int32_t reference, float* target_pose_world,
                                  float* jacobians, void* stream) {
  int st = validate_tree(tree);
  if (st) return st;
  if (batch < 0 || (batch > 0 && ((tree->nq > 0 && !q) || !jacobians))) return BR_EINVAL;  // B = 0: empty buffers
  if (!aligned4(q) || !aligned4(jacobians) || (target_pose_world && !aligned4(target_pose_world))) return BR_EALIGN;
  FkParams p = {};
  p.q = q;
  p.batch = batch;
  p.jac = jacobians;
  p.tpose = target_pose_world;
  st = fill_targets(tree, p, targets, n_targets);
  if (st) return st;
  p.outputs = OUT_JAC | (target_pose_world ? OUT_TPOSE : 0u);
  p.bulk = bulk_bit(OUT_JAC, jacobians, (int64_t)p.nt * 6 * tree->nv) |
           bulk_bit(OUT_TPOSE, target_pose_world, (int64_t)p.nt * 7);
  return dispatch_fk<true>(*tree, p, reference, (cudaStream_t)stream);
}

extern "C" int br_frame_jacobians_from_poses(const br_tree_t* tree, const float* joint_pose_world, int64_t batch,
                                             const int32_t* targets, int32_t n_targets, int32_t reference,
                                             float* jacobians, void* stream) {
  int st = validate_tree(tree);
  if (st) return st;
  if (batch < 0 || (batch > 0 && (!joint_pose_world || !jacobians))) return BR_EINVAL;  // B = 0: empty buffers
  if (!aligned4(joint_pose_world) || !aligned4(jacobians)) return BR_EALIGN;
  FkParams p = {};
  p.oMi_in = joint_pose_world;
  p.batch = batch;
  p.jac = jacobians;
  st = fill_targets(tree, p, targets, n_targets);
  if (st) return st;
  p.outputs = OUT_JAC;
  p.bulk = bulk_bit(OUT_JAC, jacobians, (int64_t)p.nt * 6 * tree->nv);
  return dispatch_fk<false>(*tree, p, reference, (cudaStream_t)stream);
}

extern "C" const char* br_version(void) { return "br_b200 0.1 (sm_100a)"; }
