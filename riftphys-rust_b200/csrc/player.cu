// player.cu -- the kinematic player controller on the device (World::update_players,
// riftphys-world/src/world/step.rs:544-639), run at the start of each tick. The players go in
// order, each seeing the poses the ones before it left, so one block runs them one after another;
// inside each of a player's (at most four) slide passes the block's threads test a chunk of
// terrain triangles, then of colliders, at once and keep the first hit in scan order, which is the
// sequential scan's answer.
#include "hf_cells.cuh"
#include "rp_narrow.cuh"
#include "shape_aabb.cuh"
#include "step_internal.cuh"

namespace rp {

namespace {
constexpr int PT = 256;  // threads of the player block
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr unsigned long long kNoHit = ~0ull;

// Aabb::intersects (riftphys-geom/src/aabb.rs:75-79)
__device__ __forceinline__ bool boxes_meet(f3 amn, f3 amx, f3 bmn, f3 bmx) {
  return amn.x <= bmx.x && amx.x >= bmn.x && amn.y <= bmx.y && amx.y >= bmn.y && amn.z <= bmx.z && amx.z >= bmn.z;
}
__device__ __forceinline__ void clear_first_point(Manifold* m) {
  m->len = 0;
  m->normal = mk3(0, 0, 0);
  m->pts[0].position = mk3(0, 0, 0);
  m->pts[0].normal = mk3(0, 0, 0);
  m->pts[0].penetration = 0.0f;
}
}  // namespace

// Body -> controller index for the bodies that carry one.
__global__ void k_player_map(uint32_t np, const PlayerGpu* __restrict__ pl, uint32_t* player_of) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < np) player_of[pl[i].body] = i;
}

// One block. Colliders' stored AABBs are the poses at the tick's start (the player pass moves its
// bodies with Bodies::set_pose, which leaves the AABBs alone), so a moved player's capsule is
// prefiltered at its start pose and tested at its new one.
__global__ void __launch_bounds__(PT) k_players(uint32_t np, PlayerGpu* pl, const uint32_t* __restrict__ player_of,
                                                float dt, uint32_t ncol, const uint32_t* __restrict__ cbody,
                                                const uint32_t* __restrict__ ckind, const float4* __restrict__ cdims,
                                                float4* pos, float4* rot, const uint8_t* __restrict__ alive,
                                                const uint8_t* __restrict__ dyn, const float* __restrict__ inv_mass,
                                                float4* lin, uint8_t* awake, uint16_t* sleep_ticks, bool has_hf,
                                                HfDev hf) {
  const int tid = threadIdx.x;
  for (uint32_t i = tid; i < np; i += PT) {
    const uint32_t b = pl[i].body;
    const float4 p = pos[b], q = rot[b];
    pl[i].p0[0] = p.x; pl[i].p0[1] = p.y; pl[i].p0[2] = p.z;
    pl[i].q0[0] = q.x; pl[i].q0[1] = q.y; pl[i].q0[2] = q.z; pl[i].q0[3] = q.w;
  }
  __shared__ f3 s_p, s_des, s_hn;
  __shared__ float s_pen;
  __shared__ uint32_t s_hbody;
  __shared__ unsigned long long s_first;
  __shared__ int s_go;
  __syncthreads();
  for (uint32_t i = 0; i < np; ++i) {
    const uint32_t body = pl[i].body;
    const float r = pl[i].radius, hh = pl[i].height * 0.5f;
    bool grounded = false;
    float vv = 0.0f;
    if (tid == 0) {
      // 1. gravity, or the sticky floor (step.rs:550-556)
      vv = pl[i].vvel;
      if (!pl[i].grounded) vv -= 9.81f * dt;
      else if (vv <= 0.0f) vv = -0.5f;
      // 2. the input direction at the player's speed (step.rs:558-567)
      const f3 in = mk3(pl[i].in[0], pl[i].in[1], pl[i].in[2]);
      const float im2 = dot(in, in);
      f3 md = mk3(0, 0, 0);
      if (im2 > 1.0e-6f) {
        const float s = sqrtf(im2);
        md = mk3(in.x / s, in.y / s, in.z / s);
      }
      const float sp = pl[i].speed;
      const f3 mv = mk3((md.x * sp) * dt, (md.y * sp) * dt, (md.z * sp) * dt);
      s_des = mk3(mv.x + 0.0f, mv.y + vv * dt, mv.z + 0.0f);
      s_p = xyz(pos[body]);
    }
    __syncthreads();
    // 3. up to four slide passes (step.rs:571-632)
    for (int it = 0; it < 4; ++it) {
      const f3 des = s_des;
      if (dot(des, des) < 1.0e-6f) break;
      const f3 xp = s_p + des;
      const q4 qid = mkq(0, 0, 0, 1);
      Shape cap;
      cap.kind = SH_CAPSULE; cap.a = r; cap.b = hh; cap.c = 0.0f;
      Iso cx;
      cx.pos = xp; cx.rot = qid;
      f3 mn, mx;
      aabb_of(SH_CAPSULE, make_float4(r, hh, 0.0f, 0.0f), xp, qid, &mn, &mx);
      if (tid == 0) s_first = kNoHit;
      __syncthreads();
      bool found = false;
      // A. the terrain triangles under the capsule's box, 5 cm of margin; the first that touches
      long long gx0, gx1, gz0, gz1;
      if (has_hf && hf_window(hf, mn, mx, &gx0, &gx1, &gz0, &gz1)) {
        const unsigned long long wx = (unsigned long long)(gx1 - gx0 + 1);
        const unsigned long long ntri = 2ull * wx * (unsigned long long)(gz1 - gz0 + 1);
        for (unsigned long long base = 0; base < ntri; base += PT) {
          const unsigned long long k = base + tid;
          Manifold m;
          clear_first_point(&m);
          if (k < ntri) {
            Tri t;
            hf_tri(hf, gx0, wx, gz0, k, &t);
            if (collide_tri(cap, cx, t, 0.05f, &m)) atomicMin(&s_first, k);
          }
          __syncthreads();
          const unsigned long long f = s_first;
          if (f != kNoHit && k == f) { s_hn = m.pts[0].normal; s_pen = m.pts[0].penetration; s_hbody = kNone; }
          __syncthreads();
          if (f != kNoHit) { found = true; break; }
        }
      }
      // B. the colliders in order, but the player's own, whose stored AABB meets the capsule's box
      if (!found) {
        for (uint32_t base = 0; base < ncol; base += PT) {
          const uint32_t ci = base + tid;
          Manifold m;
          clear_first_point(&m);
          uint32_t bd = kNone;
          if (ci < ncol) {
            bd = cbody[ci];
            if (bd != body && alive[bd]) {
              const uint32_t pj = player_of[bd];
              f3 bp;
              q4 bq;
              if (pj != kNone) {
                bp = mk3(pl[pj].p0[0], pl[pj].p0[1], pl[pj].p0[2]);
                bq = mkq(pl[pj].q0[0], pl[pj].q0[1], pl[pj].q0[2], pl[pj].q0[3]);
              } else {
                bp = xyz(pos[bd]);
                bq = asq(rot[bd]);
              }
              f3 cmn, cmx;
              aabb_of(ckind[ci], cdims[ci], bp, bq, &cmn, &cmx);
              if (boxes_meet(mn, mx, cmn, cmx)) {
                const float4 d = cdims[ci];
                Shape sh;
                sh.kind = ckind[ci]; sh.a = d.x; sh.b = d.y; sh.c = d.z;
                Iso bx;
                bx.pos = xyz(pos[bd]); bx.rot = asq(rot[bd]);
                if (collide_pair(cap, cx, sh, bx, 0.05f, &m)) atomicMin(&s_first, (unsigned long long)ci);
              }
            }
          }
          __syncthreads();
          const unsigned long long f = s_first;
          if (f != kNoHit && (unsigned long long)ci == f) {
            s_hn = m.pts[0].normal; s_pen = m.pts[0].penetration; s_hbody = bd;
          }
          __syncthreads();
          if (f != kNoHit) { found = true; break; }
        }
      }
      // C. push out of the hit and drop the motion into it; a floor grounds the player, a
      //    dynamic body is woken and kicked
      if (tid == 0) {
        f3 d2 = des;
        if (found) {
          const f3 n = s_hn;
          if (n.y > 0.6f) { grounded = true; vv = 0.0f; }
          d2 = d2 + n * (s_pen + 0.001f);
          const float dn = dot(d2, n);
          if (dn < 0.0f) d2 = d2 - n * dn;
          const uint32_t hb = s_hbody;
          if (hb != kNone && dyn[hb]) {
            awake[hb] = 1; sleep_ticks[hb] = 0;  // SleepManager::wake (sleep.rs:22-26)
            const float im = inv_mass[hb];
            const f3 j = mk3(-n.x, -n.y, -n.z) * 10.0f;
            if (im > 0.0f && vfin(j)) lin[hb] = f4(fin_v(xyz(lin[hb]) + j * im));
          }
        }
        s_des = d2;
        s_go = found ? 1 : 0;
      }
      __syncthreads();
      if (!s_go) break;
    }
    if (tid == 0) {
      // the move, through Bodies::set_pose (dynamics.rs:130-134)
      const f3 p = s_p + s_des;
      if (vfin(p)) pos[body] = f4(fin_v(p), pos[body].w);
      rot[body] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
      pl[i].vvel = vv;
      pl[i].grounded = grounded ? 1u : 0u;
    }
    __syncthreads();
  }
}

uint32_t WorldGpu::add_player(const float pose[7], float radius, float height, float speed) {
  if (batch_) throw std::invalid_argument("players act on one world; this world is a batch");
  players();  // the device's controller state first
  const float dims[3] = {0.4f, 0.9f, 0.0f};
  const float zero[6] = {0, 0, 0, 0, 0, 0};
  const uint32_t body = add_body(pose, zero, SH_CAPSULE, dims, 0.0f, zero, false, 0u, true);
  PlayerGpu p{};
  p.body = body;
  p.radius = radius; p.height = height; p.speed = speed;
  p.vvel = 0.0f; p.grounded = 0;
  h_players_.push_back(p);
  set_players(h_players_);
  return (uint32_t)h_players_.size() - 1;
}
const std::vector<PlayerGpu>& WorldGpu::players() {
  if (players_dev_newer_ && !h_players_.empty()) {
    RP_CUDA(cudaMemcpyAsync(h_players_.data(), players_d.p, sizeof(PlayerGpu) * h_players_.size(),
                            cudaMemcpyDeviceToHost, stream_));
    RP_CUDA(cudaStreamSynchronize(stream_));
  }
  players_dev_newer_ = false;
  return h_players_;
}
void WorldGpu::set_players(const std::vector<PlayerGpu>& v) {
  if (&v != &h_players_) h_players_ = v;
  players_dev_newer_ = false;
  if (h_players_.empty()) return;
  players_d.ensure(h_players_.size() + 1);
  RP_CUDA(cudaMemcpyAsync(players_d.p, h_players_.data(), sizeof(PlayerGpu) * h_players_.size(), cudaMemcpyHostToDevice,
                          stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
}
void WorldGpu::set_player_input(uint32_t i, const float dir[3]) {
  players();
  h_players_[i].in[0] = dir[0]; h_players_[i].in[1] = dir[1]; h_players_[i].in[2] = dir[2];
  set_players(h_players_);
}
void WorldGpu::get_player(uint32_t i, float pose[7], bool* grounded) {
  const PlayerGpu& p = players()[i];
  get_body_pose(p.body, pose);
  *grounded = p.grounded != 0;
}
void WorldGpu::run_players(float dt) {
  const uint32_t np = (uint32_t)h_players_.size();
  if (np == 0) return;
  cudaStream_t st = stream_;
  player_of_d.ensure(nb_ + 1);
  RP_CUDA(cudaMemsetAsync(player_of_d.p, 0xFF, 4 * (size_t)nb_, st));
  k_player_map<<<(np + PT - 1) / PT, PT, 0, st>>>(np, players_d.p, player_of_d.p); RP_COUNT_LAUNCH(1);
  HfDev hf{hf_h_.p, hf_nx_, hf_nz_, hf_sx_, hf_sz_, hf_ox_, hf_oz_, hf_min_, hf_max_};
  k_players<<<1, PT, 0, st>>>(np, players_d.p, player_of_d.p, dt, ncol_, col_body.p, col_kind.p, col_dims.p, pos.p,
                              rot.p, alive_d.p, dyn.p, inv_mass.p, lin.p, awake.p, sleep_ticks.p, has_hf_, hf);
  RP_COUNT_LAUNCH(1);
  players_dev_newer_ = true;
}

}  // namespace rp
