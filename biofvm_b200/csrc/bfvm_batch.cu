// Many independent microenvironments advanced together (libbfvm.so).
//
// A bfvm_batch holds non-owning references to bfvm_solver instances of one
// device and one precision.  bfvm_batch_step(b, dt, n, flags) has the effect
// of bfvm_step(m, dt, n, flags) on every instance: per instance the Thomas
// setup is done once from its first dt (BioFVM_solvers.cpp:87,172), and a
// step is bulk -> cells -> Dirichlet, x sweep, Dirichlet, y sweep,
// Dirichlet, z sweep (BioFVM_solvers.cpp:175-273).
//
// Scheduling.  The instances are packed, first fit in decreasing size, into
// groups whose density fields together stay within a byte budget (by
// default a fraction of the L2 cache), and all n steps of one group run
// before the next group starts: a group small enough for L2 keeps its fields
// on chip across the three sweeps of a step and from step to step.  Two
// ways to run a group (bfvm_batch_set_mode):
//   BFVM_BATCH_FUSED     every phase of a step is one launch over all of the
//                        group's instances (the kernels of
//                        bfvm_batch_kernels.cuh);
//   BFVM_BATCH_BRANCHES  every instance runs its own single-instance step
//                        kernels (its own sweep kernel choices) on a branch
//                        of its own: the branches of a group are independent
//                        graph paths that the GPU runs concurrently, so the
//                        short kernels of small instances overlap instead of
//                        running one after another.
//   BFVM_BATCH_PERSISTENT / BFVM_BATCH_PLANES
//                        all n steps of a group in one cooperative launch
//                        (bfvm_kernels_batch_steps.cuh: chunked and line
//                        forms; bfvm_kernels_batch_planes.cuh: xy planes and
//                        xz strips in shared memory); members that kernel
//                        cannot run form groups that run on branches.
// The whole sequence -- groups x steps x phases -- is captured once into a
// CUDA graph and replayed by one graph launch per call; the graph is rebuilt
// only when the plan changes (instances, their lists or device buffers, dt,
// n, flags, mode, tuning).
//
// The tuner (bfvm_batch_tune) picks, per axis, the chunk length (points per
// thread) and threads per block, then the group budget, by timing short
// graph runs on the instances' own fields, which it saves before and
// restores after.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "bfvm.h"
#include "bfvm_batch_kernels.cuh"
#include "bfvm_host_math.h"
#include "bfvm_kernels_batch_planes.cuh"
#include "bfvm_kernels_batch_steps.cuh"
#include "bfvm_state.h"

namespace bfvm_rt {
namespace {

struct BatchConfig {
  int ch[3] = {0, 0, 0};       // 0 = choose from the longest line
  int threads[3] = {0, 0, 0};  // 0 = choose
  int64_t group_bytes = -1;    // -1 = default (half of L2), 0 = one group
  int mode = BFVM_BATCH_FUSED;
  int pch = 8;  // persistent mode: points per chunk (8, 16, 32: tile form; 0: whole lines)
};

// Device descriptors of one group, all in one buffer.
struct GroupPlan {
  int64_t field_bytes = 0;
  size_t off_sweep[3] = {0, 0, 0}, off_bulk = 0, off_cells = 0, off_dir = 0;
  int n_sweep[3] = {0, 0, 0}, n_bulk = 0, n_cells = 0, n_dir = 0;
  int64_t items[3] = {0, 0, 0};
  int64_t work_bulk = 0, work_cells = 0, work_dir = 0;
  // persistent mode: the group runs as one cooperative launch over the member
  // descriptors at off_members (0: the group's members run on branches)
  int persistent = 0;
  size_t off_members = 0;
  int n_members = 0;
  int64_t ptiles[3] = {0, 0, 0};
  int64_t src_items = 0;
};

// Per-member scratch of the persistent mode: voxel maps, source and
// Dirichlet line masks, Dirichlet values at their places.
struct MemberScratch {
  DevBuf buf;
  size_t maps_bytes = 0;   // bulk_map + ag_map, set to -1 before each call
  size_t masks_off = 0, masks_bytes = 0;  // src, x, y, z masks, set to 0
  size_t dir_off = 0;      // dir_field (when the member has Dirichlet nodes)
  DevBuf tabs;             // tile form: 32-point chunk tables of the three axes
  // plane form: x-line bulk runs and their per-line offsets (rebuilt when the
  // member's lists change), per-line first sorted agents
  DevBuf runs;
  int64_t runs_version = -1;
  size_t runs_off = 0;
  DevBuf xag;
};

}  // namespace
}  // namespace bfvm_rt

struct bfvm_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<bfvm_solver*> inst;
  bfvm_rt::BatchConfig cfg;
  int l2_bytes = 0;
  // current plan
  std::vector<unsigned char> host_desc;  // descriptor bytes of every group
  std::vector<bfvm_rt::GroupPlan> groups;
  std::vector<std::vector<bfvm_solver*>> group_members;  // per group, in plan order
  int ch[3] = {16, 16, 16}, threads[3] = {256, 256, 256};
  bfvm_rt::DevBuf d_desc;
  // persistent mode: per member scratch (parallel to inst), per group the
  // host copies of the member descriptors, resident blocks per SM of the
  // 8- and 16-point kernels (0: not queried), SMs
  std::vector<bfvm_rt::MemberScratch> scratch;
  std::vector<std::vector<bfvm::StepMember>> pmembers;
  int p_per_sm[6] = {0, 0, 0, 0, 0, 0};  // 8-, 16-point chunks, line form, tile form, 4-point, planes
  size_t tile_tab_doubles = 0;  // tile form: the largest member's tables of one axis
  int num_sms = 0;
  bfvm_rt::DevBuf d_ctr;  // plane form: work-item counters, 2 per step
  // cached graph and what it was captured for
  cudaGraphExec_t exec = nullptr;
  std::string key;
  int64_t graph_kernels = 0;
};

namespace bfvm_rt {
namespace {

using namespace bfvm;

template <typename T>
void append(std::vector<unsigned char>& buf, const T& v) {
  const size_t o = buf.size();
  buf.resize(o + sizeof(T));
  std::memcpy(buf.data() + o, &v, sizeof(T));
}

void align_to(std::vector<unsigned char>& buf, size_t a) {
  buf.resize((buf.size() + a - 1) / a * a, 0);
}

int axis_len(const bfvm_solver* m, int a) { return a == 0 ? m->nx : (a == 1 ? m->ny : m->nz); }

// Chunk length and threads per block valid for every instance: a work item
// holds all chunks of its lines, at least 32 columns wide.
bool config_fits(const bfvm_batch* b, int a, int ch, int threads) {
  if (threads > batch_max_threads(ch)) return false;
  for (const bfvm_solver* m : b->inst) {
    const int nc = (axis_len(m, a) + ch - 1) / ch;
    if (nc * 32 > threads) return false;
  }
  return true;
}

void choose_shapes(bfvm_batch* b) {
  for (int a = 0; a < 3; ++a) {
    int ch = b->cfg.ch[a], th = b->cfg.threads[a];
    if (ch && th) {
      require(config_fits(b, a, ch, th),
              "batch config: chunk " + std::to_string(ch) + " x " + std::to_string(th) +
                  " threads cannot hold the longest line of axis " + std::to_string(a));
    } else {
      ch = 0;
      for (int c : {16, 32, 8})
        for (int t : {256, 512})
          if (!ch && config_fits(b, a, c, t)) ch = c, th = t;
      require(ch != 0, "batch: an axis is longer than 512 x 32 points");
    }
    b->ch[a] = ch;
    b->threads[a] = th;
  }
}

template <typename T>
BatchSweep<T> sweep_desc(const bfvm_solver* m, int a, int ch, int threads, int64_t first) {
  BatchSweep<T> d;
  std::memset(&d, 0, sizeof d);  // the bytes also key the graph cache
  const int64_t nx = m->nx, ny = m->ny, nz = m->nz, S = m->S;
  d.p = m->p.as<T>();
  d.coef = coef_view<T>(m, a);
  d.S = m->S;
  if (a == 0) {
    d.n = (int)nx;
    d.C = S;
    d.outer_stride = nx * S;
    d.line_stride = S;
    d.ncols = ny * nz * S;
  } else if (a == 1) {
    d.n = (int)ny;
    d.C = nx * S;
    d.outer_stride = nx * ny * S;
    d.line_stride = nx * S;
    d.ncols = nz * nx * S;
  } else {
    d.n = (int)nz;
    d.C = nx * ny * S;
    d.outer_stride = 0;
    d.line_stride = nx * ny * S;
    d.ncols = nx * ny * S;
  }
  d.nchunks = (d.n + ch - 1) / ch;
  d.tw = std::max(32, threads / d.nchunks / 32 * 32);
  d.first = first;
  return d;
}

// Instances packed into groups of at most `budget` field bytes, first fit
// in decreasing size (a single instance larger than the budget is a group
// of its own): small instances share groups, so that a group's members can
// run side by side.  Members are independent, so the order is free.
std::vector<std::vector<bfvm_solver*>> make_groups(const std::vector<bfvm_solver*>& inst,
                                                   int64_t budget) {
  std::vector<std::vector<bfvm_solver*>> g;
  if (inst.empty()) return g;
  if (budget <= 0) {
    g.push_back(inst);
    return g;
  }
  std::vector<bfvm_solver*> order(inst);
  auto bytes = [](const bfvm_solver* m) { return (int64_t)(m->NS() * m->elem()); };
  std::stable_sort(order.begin(), order.end(),
                   [&](const bfvm_solver* x, const bfvm_solver* y) { return bytes(x) > bytes(y); });
  std::vector<int64_t> used;
  for (bfvm_solver* m : order) {
    size_t k = 0;
    while (k < g.size() && used[k] + bytes(m) > budget) ++k;
    if (k == g.size()) {
      g.emplace_back();
      used.push_back(0);
    }
    g[k].push_back(m);
    used[k] += bytes(m);
  }
  return g;
}

// Whether a member can run in the persistent mode's kernel: FP64 field,
// lines of at most 128 points.
// (The tile form stages a member's chunk tables of one axis in shared
// memory, about 4.2 KB per density: at most 32 densities there.)
bool persistent_ok(const bfvm_solver* m, int pch) {
  return m->precision == BFVM_FP64 && m->nx <= kBatchStepsMaxN && m->ny <= kBatchStepsMaxN &&
         m->nz <= kBatchStepsMaxN && (pch != 32 || m->S <= 32);
}

// The persistent kernel's form: the chunk length of BFVM_BATCH_PERSISTENT
// (0: whole lines), or kPlaneForm for BFVM_BATCH_PLANES.
constexpr int kPlaneForm = -1;
bool persistent_mode(int mode) {
  return mode == BFVM_BATCH_PERSISTENT || mode == BFVM_BATCH_PLANES;
}
int pform(const bfvm_batch* b) { return b->cfg.mode == BFVM_BATCH_PLANES ? kPlaneForm : b->cfg.pch; }

// Plane form shapes of member m: densities per xy item (sg, balanced over
// the plane's items) and columns per z item (cw); false when even one
// density's xy plane, or one column of nz points, exceeds the block's shared
// memory.
bool plane_shape(const bfvm_solver* m, int* sg_out, int* groups_out, int* cw_out,
                 int* strips_out) {
  const int nx = m->nx, ny = m->ny, nz = m->nz, S = m->S;
  auto fits = [&](int sg) {
    return (int64_t)ny * plane_pitch(nx, sg) <= kPlaneSmemDoubles &&
           (int64_t)(nx + ny) * sg <= kPlaneTabPairs;
  };
  int sg = S;
  while (sg > 0 && !fits(sg)) --sg;
  if (sg == 0) return false;
  int groups = (S + sg - 1) / sg;
  sg = (S + groups - 1) / groups;  // the same items, balanced
  // the last item of a plane has S - (groups - 1)*sg densities; its pitch
  // rounds up on its own
  if (!fits(S - (groups - 1) * sg)) return false;
  const int C = nx * S;
  const int most = kPlaneSmemDoubles / nz;
  if (most < 1) return false;
  const int strips = (C + most - 1) / most;
  *sg_out = sg;
  *groups_out = groups;
  *cw_out = (C + strips - 1) / strips;
  *strips_out = strips;
  return true;
}

// Whether a member can run in the plane form: FP64, lines of at most 128
// points (two mask words per line), plane items that fit shared memory, and
// offsets of 32 bits inside the member.
bool planes_ok(const bfvm_solver* m) {
  int a, b, c, d;
  return m->precision == BFVM_FP64 && m->nx <= kBatchStepsMaxN && m->ny <= kBatchStepsMaxN &&
         m->nz <= kBatchStepsMaxN && m->S <= 4096 && m->NS() < ((int64_t)1 << 31) &&
         plane_shape(m, &a, &b, &c, &d);
}

bool form_ok(const bfvm_solver* m, int form) {
  return form == kPlaneForm ? planes_ok(m) : persistent_ok(m, form);
}

size_t round256(size_t x) { return (x + 255) / 256 * 256; }

// The persistent mode's descriptor of member m (device pointers into its
// scratch, which is sized here), with its first work items in each phase.
bfvm::StepMember step_member(bfvm_batch* b, bfvm_solver* m, int flags, int ch,
                             const int64_t* tile0, int64_t src0) {
  const size_t k = std::find(b->inst.begin(), b->inst.end(), m) - b->inst.begin();
  if (b->scratch.size() < b->inst.size()) b->scratch.resize(b->inst.size());
  MemberScratch& sc = b->scratch[k];
  const int64_t N = m->N();
  const int64_t lx = N / m->nx, ly = N / m->ny, lz = N / m->nz;
  sc.maps_bytes = round256((size_t)2 * N * sizeof(int));
  sc.masks_off = sc.maps_bytes;
  sc.masks_bytes = round256((size_t)2 * (lz + lx + ly + lz) * sizeof(unsigned long long));
  sc.dir_off = sc.masks_off + sc.masks_bytes;
  const size_t dir_bytes = m->dir_unique > 0 ? (size_t)N * m->S * sizeof(double) : 0;
  sc.buf.ensure(sc.dir_off + std::max<size_t>(dir_bytes, 256));
  unsigned char* base = sc.buf.as<unsigned char>();
  auto* masks = reinterpret_cast<unsigned long long*>(base + sc.masks_off);

  bfvm::StepMember d;
  std::memset(&d, 0, sizeof d);  // the bytes also key the graph cache
  d.p = m->p.as<double>();
  d.nx = m->nx;
  d.ny = m->ny;
  d.nz = m->nz;
  d.S = m->S;
  const int ns[3] = {m->nx, m->ny, m->nz};
  for (int a = 0; a < 3; ++a) {
    // ch = 0: the line form, one column per work item; ch = 32: the tile
    // form, 32 columns per work item; kPlaneForm: planes (below)
    d.nc[a] = ch > 0 ? (ns[a] + ch - 1) / ch : 1;
    d.tw[a] = ch == 32 ? kBatchTileCols : (ch > 0 ? kBatchStepsThreads / d.nc[a] : 1);
    d.ncols[a] = N / ns[a] * m->S;
    d.tile0[a] = tile0[a];
    d.coef[a] = coef_view<double>(m, a);
  }
  d.bulk = (flags & BFVM_STEP_BULK) && !m->bulk_vox.empty();
  d.cells = (flags & BFVM_STEP_CELLS) && m->n_agents > 0;
  d.dirichlet = m->dir_unique > 0;
  d.src0 = src0;
  d.nsrc = ((d.bulk ? (int64_t)m->bulk_vox.size() : 0) + (d.cells ? m->n_agents : 0)) * m->S;
  d.bulk_map = reinterpret_cast<const int*>(base);
  d.ag_map = d.bulk_map + N;
  d.src_mask = masks;
  d.dir_mask[0] = masks + 2 * lz;
  d.dir_mask[1] = masks + 2 * (lz + lx);
  d.dir_mask[2] = masks + 2 * (lz + lx + ly);
  d.dir_field = reinterpret_cast<const double*>(base + sc.dir_off);
  d.nbulk = (int64_t)m->bulk_vox.size();
  d.bulk_vox = m->d_bulk_vox.as<int64_t>();
  if (m->bulk_rows > 0) {  // shared rate rows: [rows][S][2]
    d.st = m->d_bulk_tab.as<double>();
    d.su = d.st + 1;
    d.rs = 2;
    d.bulk_row = m->d_bulk_row.as<int>();
  } else {
    d.st = m->d_bulk_st.as<double>();
    d.su = m->d_bulk_su.as<double>();
    d.rs = 1;
    d.bulk_row = nullptr;
  }
  if (ch == 32 || ch == kPlaneForm) {
    // the sweep kernels' chunk tables for 32-point chunks, every chunk its
    // own slot, from the FP64 Thomas coefficients (the plane form reads
    // their {1/d, a} pairs, [point][density], as whole-line tables)
    std::vector<double> all;
    size_t off[3][3];
    for (int a = 0; a < 3; ++a) {
      const int n = ns[a], S = m->S, nc = (n + 31) / 32;
      std::vector<double> k1((size_t)nc * 32 * S * 2), kg(k1.size()), kc((size_t)nc * S * 4);
      bfvm::chunk_tables(n, S, 32, m->h_c1[a].data(), m->h_den[a].data(), m->h_cx[a].data(),
                         k1.data(), kg.data(), kc.data());
      off[a][0] = all.size();
      all.insert(all.end(), k1.begin(), k1.end());
      off[a][1] = all.size();
      all.insert(all.end(), kg.begin(), kg.end());
      off[a][2] = all.size();
      all.insert(all.end(), kc.begin(), kc.end());
      all.resize((all.size() + 1) & ~(size_t)1, 0.0);  // 16-byte aligned sections
      b->tile_tab_doubles = std::max(b->tile_tab_doubles, all.size() - off[a][0]);
    }
    upload(sc.tabs, all, b->stream);
    const double* t = sc.tabs.as<double>();
    for (int a = 0; a < 3; ++a) {
      d.ck1[a] = t + off[a][0];
      d.ckg[a] = t + off[a][1];
      d.ckc[a] = t + off[a][2];
    }
  }
  d.nagents = m->n_agents;
  d.ag_key = m->d_ag_key.as<uint64_t>();
  d.ag_idx = m->d_ag_idx.as<int>();
  d.ag_t1 = m->d_ag_t1.as<double>();
  d.ag_t2 = m->d_ag_t2.as<double>();
  if (ch == kPlaneForm) {
    require(plane_shape(m, &d.psg, &d.pgroups, &d.pcw, &d.pstrips),
            "batch: member does not fit the plane form", BFVM_ERR_STATE);
    const int64_t lines = (int64_t)m->ny * m->nz;
    if (d.bulk && (sc.runs_version != m->lists_version || !sc.runs.ptr)) {
      // runs of consecutive voxels of one x line whose rates are bitwise
      // equal, the offsets of each line's runs after them
      const int S = m->S;
      const int64_t E = (int64_t)m->bulk_vox.size();
      std::vector<int> runs, off((size_t)lines + 1, 0);
      auto same = [&](int64_t a, int64_t c) {
        return std::memcmp(&m->bulk_st[a * S], &m->bulk_st[c * S], S * sizeof(double)) == 0 &&
               std::memcmp(&m->bulk_su[a * S], &m->bulk_su[c * S], S * sizeof(double)) == 0;
      };
      int64_t first = 0;
      for (int64_t e = 0; e < E; ++e) {
        const int64_t v = m->bulk_vox[e];
        const bool open = e > 0 && v == m->bulk_vox[e - 1] + 1 && v / m->nx == (v - 1) / m->nx &&
                          same(first, e);
        if (open) {
          runs[runs.size() - 3] += 1;  // end x
          continue;
        }
        first = e;
        const int64_t line = v / m->nx;
        const int x = (int)(v - line * m->nx);
        runs.push_back(x);
        runs.push_back(x + 1);
        runs.push_back((int)e);
        runs.push_back(0);
        off[(size_t)line + 1] += 1;
      }
      for (size_t i = 1; i < off.size(); ++i) off[i] += off[i - 1];
      sc.runs_off = round256(runs.size() * sizeof(int));
      sc.runs.ensure(sc.runs_off + off.size() * sizeof(int));
      if (!runs.empty())
        BFVM_CUDA(cudaMemcpyAsync(sc.runs.ptr, runs.data(), runs.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, b->stream));
      BFVM_CUDA(cudaMemcpyAsync(sc.runs.as<unsigned char>() + sc.runs_off, off.data(),
                                off.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream));
      sc.runs_version = m->lists_version;
    }
    if (d.bulk) {
      d.xruns = sc.runs.as<int4>();
      d.xrun_off = reinterpret_cast<const int*>(sc.runs.as<unsigned char>() + sc.runs_off);
      d.est = m->d_bulk_st.as<double>();
      d.esu = m->d_bulk_su.as<double>();
    }
    if (d.cells) {
      sc.xag.ensure((size_t)(lines + 1) * sizeof(int));
      d.xag_off = sc.xag.as<int>();
    }
  }
  return d;
}

template <typename T>
void build_plan(bfvm_batch* b, int flags) {
  const int64_t budget = b->cfg.group_bytes < 0 ? (int64_t)b->l2_bytes / 2 : b->cfg.group_bytes;
  // persistent mode (FP64, whole steps): the members its kernel can run form
  // groups of their own, run first; the others run on branches
  std::vector<bfvm_solver*> pers, rest;
  const bool persistent = persistent_mode(b->cfg.mode) && sizeof(T) == sizeof(double) &&
                          (flags & BFVM_STEP_DIFFUSION);
  const int form = pform(b);
  for (bfvm_solver* m : b->inst) (persistent && form_ok(m, form) ? pers : rest).push_back(m);
  auto pgroups = make_groups(pers, budget);
  const size_t n_pers = pgroups.size();
  auto groups = pgroups;
  for (auto& g : make_groups(rest, budget)) groups.push_back(g);
  std::vector<unsigned char>& buf = b->host_desc;
  buf.clear();
  b->groups.clear();
  b->pmembers.clear();
  b->tile_tab_doubles = 0;
  b->group_members = groups;
  for (size_t gi = 0; gi < groups.size(); ++gi) {
    auto& members = groups[gi];
    GroupPlan G;
    std::memset(&G, 0, sizeof G);
    for (bfvm_solver* m : members) G.field_bytes += (int64_t)(m->NS() * m->elem());
    if (gi < n_pers) {
      G.persistent = 1;
      std::vector<bfvm::StepMember> ds;
      int64_t tile0[3] = {0, 0, 0}, src0 = 0;
      for (bfvm_solver* m : members) {
        bfvm::StepMember d = step_member(b, m, flags, form, tile0, src0);
        if (form == kPlaneForm) {
          // xy items: every plane's density groups; z items: every xz
          // plane's strips
          tile0[0] += (int64_t)m->nz * d.pgroups;
          tile0[2] += (int64_t)m->ny * d.pstrips;
        } else {
          for (int a = 0; a < 3; ++a) tile0[a] += (d.ncols[a] + d.tw[a] - 1) / d.tw[a];
        }
        src0 += d.nsrc;
        ds.push_back(d);
      }
      align_to(buf, 64);
      G.off_members = buf.size();
      for (const auto& d : ds) append(buf, d);
      G.n_members = (int)ds.size();
      for (int a = 0; a < 3; ++a) G.ptiles[a] = tile0[a];
      G.src_items = src0;
      b->pmembers.push_back(ds);
      b->groups.push_back(G);
      continue;
    }
    b->pmembers.emplace_back();
    for (int a = 0; a < 3; ++a) {
      align_to(buf, 64);
      G.off_sweep[a] = buf.size();
      int64_t first = 0;
      for (bfvm_solver* m : members) {
        BatchSweep<T> d = sweep_desc<T>(m, a, b->ch[a], b->threads[a], first);
        if (d.ncols == 0) continue;
        first += (d.ncols + d.tw - 1) / d.tw;
        append(buf, d);
        G.n_sweep[a]++;
      }
      G.items[a] = first;
    }
    auto lists = [&](size_t& off, int& n, int64_t& work, auto fill) {
      align_to(buf, 64);
      off = buf.size();
      for (bfvm_solver* m : members) {
        BatchList<T> L;
        std::memset(&L, 0, sizeof L);
        L.p = m->p.as<T>();
        L.S = m->S;
        if (!fill(m, L) || L.count == 0) continue;
        L.first = work;
        work += L.count * m->S;
        append(buf, L);
        n++;
      }
    };
    lists(G.off_bulk, G.n_bulk, G.work_bulk, [](bfvm_solver* m, BatchList<T>& L) {
      L.count = (int64_t)m->bulk_vox.size();
      L.vox = m->d_bulk_vox.as<int64_t>();
      L.a = m->d_bulk_st.as<double>();
      L.b = m->d_bulk_su.as<double>();
      return true;
    });
    lists(G.off_cells, G.n_cells, G.work_cells, [](bfvm_solver* m, BatchList<T>& L) {
      L.count = m->n_agents;
      L.key = m->d_ag_key.as<uint64_t>();
      L.idx = m->d_ag_idx.as<int>();
      L.a = m->d_ag_t1.as<double>();
      L.b = m->d_ag_t2.as<double>();
      return true;
    });
    lists(G.off_dir, G.n_dir, G.work_dir, [](bfvm_solver* m, BatchList<T>& L) {
      L.count = m->dir_unique;
      L.vox = m->d_dir_vox.as<int64_t>();
      L.a = m->d_dir_val.as<double>();
      return true;
    });
    b->groups.push_back(G);
  }
  align_to(buf, 64);
}

template <typename T>
void launch_sweep_group(bfvm_batch* b, const GroupPlan& G, int a, int64_t* kernels) {
  if (G.items[a] == 0) return;
  const auto* sw = reinterpret_cast<const BatchSweep<T>*>(b->d_desc.as<unsigned char>() +
                                                          G.off_sweep[a]);
  const int th = b->threads[a];
  const size_t smem = 4 * sizeof(T) * (size_t)th;
  const dim3 grid((unsigned)G.items[a]);
  switch (b->ch[a]) {
    case 8: lod_batch_sweep_kernel<T, 8><<<grid, th, smem, b->stream>>>(sw, G.n_sweep[a]); break;
    case 16: lod_batch_sweep_kernel<T, 16><<<grid, th, smem, b->stream>>>(sw, G.n_sweep[a]); break;
    case 32: lod_batch_sweep_kernel<T, 32><<<grid, th, smem, b->stream>>>(sw, G.n_sweep[a]); break;
    default: throw Error(BFVM_ERR_STATE, "unsupported batch chunk length");
  }
  BFVM_CUDA(cudaGetLastError());
  ++*kernels;
}

template <typename T>
void launch_dirichlet_group(bfvm_batch* b, const GroupPlan& G, int64_t* kernels) {
  if (G.work_dir == 0) return;
  const auto* L =
      reinterpret_cast<const BatchList<T>*>(b->d_desc.as<unsigned char>() + G.off_dir);
  batch_dirichlet_kernel<T><<<(unsigned)blocks_for(G.work_dir, 256), 256, 0, b->stream>>>(
      L, G.n_dir, G.work_dir);
  BFVM_CUDA(cudaGetLastError());
  ++*kernels;
}

// One step of one group; `axes` limits the sweeps (the tuner times one axis).
template <typename T>
void enqueue_group_step(bfvm_batch* b, const GroupPlan& G, double dt, int flags, int axes,
                        int64_t* kernels) {
  unsigned char* base = b->d_desc.as<unsigned char>();
  if ((flags & BFVM_STEP_BULK) && G.work_bulk) {
    const auto* L = reinterpret_cast<const BatchList<T>*>(base + G.off_bulk);
    batch_bulk_kernel<T><<<(unsigned)blocks_for(G.work_bulk, 256), 256, 0, b->stream>>>(
        L, G.n_bulk, G.work_bulk, dt);
    BFVM_CUDA(cudaGetLastError());
    ++*kernels;
  }
  if ((flags & BFVM_STEP_CELLS) && G.work_cells) {
    const auto* L = reinterpret_cast<const BatchList<T>*>(base + G.off_cells);
    batch_cells_kernel<T><<<(unsigned)blocks_for(G.work_cells, 256), 256, 0, b->stream>>>(
        L, G.n_cells, G.work_cells);
    BFVM_CUDA(cudaGetLastError());
    ++*kernels;
  }
  if (!(flags & BFVM_STEP_DIFFUSION)) return;
  for (int a = 0; a < 3; ++a) {
    if (!(axes & (1 << a))) continue;
    launch_dirichlet_group<T>(b, G, kernels);
    launch_sweep_group<T>(b, G, a, kernels);
  }
}

// Dynamic shared memory above the default 48 KB for a persistent kernel.
void allow_persistent_smem(const void* k, size_t smem) {
  if (smem > 48 * 1024)
    BFVM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
}

// Resident blocks per SM of the persistent kernel with ch-point chunks
// (queried once per batch).
// The persistent kernel for chunk length ch (0: the line form) and its
// dynamic shared memory.
const void* persistent_kernel(const bfvm_batch* b, int ch, size_t* smem) {
  if (ch == kPlaneForm) {
    *smem = (size_t)kPlaneSmemDoubles * sizeof(double) + (size_t)kPlaneTabPairs * 16;
    return (const void*)batch_planes_kernel;
  }
  *smem = ch == 32 ? 4 * kBatchTileCols * sizeof(bfvm::Pair<double>) +
                         b->tile_tab_doubles * sizeof(double)
                   : (ch > 0 ? 4 * kBatchStepsThreads * sizeof(double) : 0);
  if (ch == 4) return (const void*)batch_steps_kernel<4>;
  if (ch == 8) return (const void*)batch_steps_kernel<8>;
  if (ch == 16) return (const void*)batch_steps_kernel<16>;
  if (ch == 32) return (const void*)batch_tiles_kernel;
  return (const void*)batch_lines_kernel<kBatchLineBatch>;
}

int persistent_threads(int ch) { return ch == kPlaneForm ? kPlaneThreads : kBatchStepsThreads; }

int persistent_per_sm(bfvm_batch* b, int ch) {
  const int i = ch == kPlaneForm
                    ? 5
                    : (ch == 8 ? 0 : (ch == 16 ? 1 : (ch == 0 ? 2 : (ch == 32 ? 3 : 4))));
  if (b->p_per_sm[i] == 0 || i == 3) {  // the tile form's shared memory varies
    int coop = 0;
    BFVM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, b->device));
    require(coop != 0, "batch: the device cannot launch cooperative kernels", BFVM_ERR_CUDA);
    BFVM_CUDA(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device));
    size_t smem = 0;
    const void* k = persistent_kernel(b, ch, &smem);
    allow_persistent_smem(k, smem);
    int per = 0;
    BFVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, persistent_threads(ch), smem));
    require(per > 0, "batch: the persistent kernel cannot be resident", BFVM_ERR_CUDA);
    b->p_per_sm[i] = per;
  }
  return b->p_per_sm[i];
}

// Blocks of a persistent group's launch: enough for the widest phase, at
// most one wave of resident blocks (every block must be resident).
int persistent_blocks(bfvm_batch* b, const GroupPlan& G) {
  const int form = pform(b);
  const int64_t wave = (int64_t)persistent_per_sm(b, form) * b->num_sms;
  const int th = persistent_threads(form);
  int64_t want = (G.src_items + th - 1) / th;
  for (int a = 0; a < 3; ++a)
    want = std::max(want, form != 0 ? G.ptiles[a] : (G.ptiles[a] + th - 1) / th);
  return (int)std::max<int64_t>(1, std::min(want, wave));
}

// A persistent group: every member's maps, then all nsteps steps of all
// members in one cooperative launch.
void enqueue_persistent_group(bfvm_batch* b, size_t gi, double dt, int nsteps,
                              int64_t* kernels) {
  const GroupPlan& G = b->groups[gi];
  const std::vector<bfvm_solver*>& members = b->group_members[gi];
  const std::vector<bfvm::StepMember>& ds = b->pmembers[gi];
  bool sources = false;
  for (size_t k = 0; k < members.size(); ++k) {
    bfvm_solver* m = members[k];
    const bfvm::StepMember& d = ds[k];
    const size_t idx = std::find(b->inst.begin(), b->inst.end(), m) - b->inst.begin();
    MemberScratch& sc = b->scratch[idx];
    unsigned char* base = sc.buf.as<unsigned char>();
    sources = sources || d.bulk || d.cells;
    if (pform(b) == kPlaneForm) {
      if (d.cells) {  // the x lines' first sorted agents
        const int64_t lines = (int64_t)m->ny * m->nz;
        plane_agent_lines_kernel<<<(unsigned)blocks_for(lines + 1, 256), 256, 0, b->stream>>>(
            d, const_cast<int*>(d.xag_off));
        BFVM_CUDA(cudaGetLastError());
        ++*kernels;
      }
      // the plane form reads only the Dirichlet masks and values of the maps
      if (!d.dirichlet) continue;
    } else if (!d.bulk && !d.cells && !d.dirichlet) {
      continue;
    }
    BFVM_CUDA(cudaMemsetAsync(base, 0xFF, sc.maps_bytes, b->stream));
    BFVM_CUDA(cudaMemsetAsync(base + sc.masks_off, 0, sc.masks_bytes, b->stream));
    const int64_t most = std::max({d.bulk ? d.nbulk : 0, d.cells ? d.nagents : 0, m->dir_unique});
    if (most == 0) continue;
    bfvm::StepMember dm = d;
    if (!d.bulk) dm.nbulk = 0;
    if (!d.cells) dm.nagents = 0;
    batch_maps_kernel<<<(unsigned)blocks_for(most, 256), 256, 0, b->stream>>>(
        dm, m->d_dir_vox.as<int64_t>(), m->d_dir_val.as<double>(), m->dir_unique,
        reinterpret_cast<int*>(base), reinterpret_cast<int*>(base) + m->N(),
        const_cast<unsigned long long*>(d.src_mask), const_cast<unsigned long long*>(d.dir_mask[0]),
        const_cast<unsigned long long*>(d.dir_mask[1]),
        const_cast<unsigned long long*>(d.dir_mask[2]), const_cast<double*>(d.dir_field));
    BFVM_CUDA(cudaGetLastError());
    ++*kernels;
  }
  bfvm::BatchStepsArgs a;
  std::memset(&a, 0, sizeof a);
  a.mem = reinterpret_cast<const bfvm::StepMember*>(b->d_desc.as<unsigned char>() + G.off_members);
  a.nmem = G.n_members;
  for (int ax = 0; ax < 3; ++ax) a.tiles[ax] = G.ptiles[ax];
  a.src_items = G.src_items;
  a.nsteps = nsteps;
  a.dt = dt;
  a.sources = sources ? 1 : 0;
  const int form = pform(b);
  if (form == kPlaneForm) {
    // the phases' work-item counters start at zero for every launch
    const size_t bytes = (size_t)2 * nsteps * sizeof(int);
    require(b->d_ctr.bytes >= bytes, "batch: work-item counters not sized", BFVM_ERR_STATE);
    a.ctr = b->d_ctr.as<int>();
    BFVM_CUDA(cudaMemsetAsync(a.ctr, 0, bytes, b->stream));
  }
  const int blocks = persistent_blocks(b, G);
  size_t smem = 0;
  const void* kern = persistent_kernel(b, form, &smem);
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(persistent_threads(form));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* params[] = {&a};
  BFVM_CUDA(cudaLaunchKernelExC(&cfg, kern, params));
  ++*kernels;
}

// Makes every instance ready for a step (Thomas setup from this dt when not
// yet done, lists on the device) and orders the batch stream after the work
// already queued on the instances' own streams.
void prepare_instances(bfvm_batch* b, double dt) {
  for (bfvm_solver* m : b->inst) {
    DeviceGuard dg(m->device);
    check_lod_mesh(m);
    require(m->lod_dims == 3, "batch: instance is inside a LOD_2D step", BFVM_ERR_STATE);
    if (!m->setup_done) thomas_setup(m, dt);
    build_all(m);
    BFVM_CUDA(cudaEventRecord(b->ev, m->stream));
    BFVM_CUDA(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
}

// Later work on the instances' streams waits for the batch.
void release_instances(bfvm_batch* b) {
  BFVM_CUDA(cudaEventRecord(b->ev, b->stream));
  for (bfvm_solver* m : b->inst) BFVM_CUDA(cudaStreamWaitEvent(m->stream, b->ev, 0));
}

bool fp64(const bfvm_batch* b) { return b->inst.empty() || b->inst[0]->precision == BFVM_FP64; }

void plan(bfvm_batch* b, int flags) {
  choose_shapes(b);
  if (fp64(b))
    build_plan<double>(b, flags);
  else
    build_plan<float>(b, flags);
  // the persistent kernel's shared-memory limit and occupancy, settled here,
  // outside any graph capture
  bool any_persistent = false;
  for (const GroupPlan& G : b->groups) any_persistent = any_persistent || G.persistent;
  if (any_persistent) persistent_per_sm(b, pform(b));
  b->d_desc.ensure(std::max<size_t>(b->host_desc.size(), 64));
  BFVM_CUDA(cudaMemcpyAsync(b->d_desc.ptr, b->host_desc.data(), b->host_desc.size(),
                            cudaMemcpyHostToDevice, b->stream));
}

void drop_graph(bfvm_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->key.clear();
}

// Branch mode: one step of one instance with its own kernels, on its own
// stream (bfvm_step's statements).  `axes` limits the sweeps as above.
void enqueue_instance_step(bfvm_solver* m, double dt, int flags, int axes) {
  if (!(flags & BFVM_STEP_DIFFUSION)) {
    if (flags & BFVM_STEP_BULK) bulk_any(m, dt);
    if (flags & BFVM_STEP_CELLS) cells_any(m);
    return;
  }
  if (axes == 7) {
    step_once(m, dt, flags, nullptr);
    return;
  }
  const int fuses[3] = {kFuseDirPro | kFuseDirEpi, kFuseDirEpi, 0};
  for (int a = 0; a < 3; ++a)
    if (axes & (1 << a)) sweep(m, a, fuses[a], dt);
}

// Branch mode: runs one step of every instance outside any capture, on its
// field saved before and restored after, so that everything a step prepares
// on first use (coefficient and chunk tables, kernel attributes) exists
// before the capture, which must not upload or synchronise.
void warm_instances(bfvm_batch* b, double dt, int flags) {
  std::vector<bfvm_solver*> on_branches;
  for (size_t gi = 0; gi < b->groups.size(); ++gi)
    if (!b->groups[gi].persistent)
      on_branches.insert(on_branches.end(), b->group_members[gi].begin(),
                         b->group_members[gi].end());
  for (bfvm_solver* m : on_branches) {
    const size_t bytes = m->NS() * m->elem();
    if (bytes == 0) continue;
    DevBuf save;
    save.ensure(bytes);
    BFVM_CUDA(cudaMemcpyAsync(save.ptr, m->p.ptr, bytes, cudaMemcpyDeviceToDevice, m->stream));
    enqueue_instance_step(m, dt, flags, 7);
    BFVM_CUDA(cudaMemcpyAsync(m->p.ptr, save.ptr, bytes, cudaMemcpyDeviceToDevice, m->stream));
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
    check_status(m);
  }
}

// Captures groups x nsteps x phases into one graph executable.
cudaGraphExec_t capture(bfvm_batch* b, double dt, int nsteps, int flags, int axes,
                        int64_t* kernels) {
  *kernels = 0;
  cudaGraph_t graph = nullptr;
  // branch mode, and the persistent modes' groups that their kernel cannot run
  const bool branches = b->cfg.mode == BFVM_BATCH_BRANCHES || persistent_mode(b->cfg.mode);
  if (branches) warm_instances(b, dt, flags);
  if (b->cfg.mode == BFVM_BATCH_PLANES) b->d_ctr.ensure((size_t)2 * std::max(nsteps, 1) * sizeof(int));
  BFVM_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  try {
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
      const GroupPlan& G = b->groups[gi];
      if (G.persistent) {
        if (axes != 7) throw Error(BFVM_ERR_STATE, "persistent groups run whole steps");
        enqueue_persistent_group(b, gi, dt, nsteps, kernels);
        continue;
      }
      if (branches) {
        // fork: every member's own stream joins the capture after the work
        // captured so far; join: the batch stream waits for every member
        const std::vector<bfvm_solver*>& members = b->group_members[gi];
        BFVM_CUDA(cudaEventRecord(b->ev, b->stream));
        for (bfvm_solver* m : members) BFVM_CUDA(cudaStreamWaitEvent(m->stream, b->ev, 0));
        for (bfvm_solver* m : members) {
          const int64_t before = m->launches;
          for (int it = 0; it < nsteps; ++it) enqueue_instance_step(m, dt, flags, axes);
          *kernels += m->launches - before;
        }
        for (bfvm_solver* m : members) {
          BFVM_CUDA(cudaEventRecord(b->ev, m->stream));
          BFVM_CUDA(cudaStreamWaitEvent(b->stream, b->ev, 0));
        }
        continue;
      }
      for (int it = 0; it < nsteps; ++it) {
        if (fp64(b))
          enqueue_group_step<double>(b, G, dt, flags, axes, kernels);
        else
          enqueue_group_step<float>(b, G, dt, flags, axes, kernels);
      }
    }
  } catch (...) {
    cudaStreamEndCapture(b->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  BFVM_CUDA(cudaStreamEndCapture(b->stream, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  BFVM_CUDA(e);
  return exec;
}

std::string plan_key(const bfvm_batch* b, double dt, int nsteps, int flags) {
  std::string k(reinterpret_cast<const char*>(b->host_desc.data()), b->host_desc.size());
  k.append(reinterpret_cast<const char*>(&dt), sizeof dt);
  k.append(reinterpret_cast<const char*>(&nsteps), sizeof nsteps);
  k.append(reinterpret_cast<const char*>(&flags), sizeof flags);
  k.append(reinterpret_cast<const char*>(b->ch), sizeof b->ch);
  k.append(reinterpret_cast<const char*>(b->threads), sizeof b->threads);
  k.append(reinterpret_cast<const char*>(&b->cfg.mode), sizeof b->cfg.mode);
  k.append(reinterpret_cast<const char*>(&b->cfg.pch), sizeof b->cfg.pch);
  // branch mode (and the persistent mode's groups on branches) bakes each
  // member's own kernel choices and device buffers into the graph
  if (b->cfg.mode == BFVM_BATCH_BRANCHES || persistent_mode(b->cfg.mode))
    for (const bfvm_solver* m : b->inst) {
      for (int a = 0; a < 3; ++a) {
        const Axis& A = m->axis[a];
        const int v[5] = {A.ch, A.tw, A.minb, A.kind, m->chunk_nslots[a]};
        k.append(reinterpret_cast<const char*>(v), sizeof v);
      }
      const int64_t v[8] = {m->path, m->fuse_sources, m->precision, m->n_agents,
                            (int64_t)m->bulk_vox.size(), m->dir_unique, m->NS(), m->S};
      k.append(reinterpret_cast<const char*>(v), sizeof v);
      auto buf = [&](const DevBuf& d) {
        k.append(reinterpret_cast<const char*>(&d.ptr), sizeof d.ptr);
        k.append(reinterpret_cast<const char*>(&d.bytes), sizeof d.bytes);
      };
      auto seg = [&](const DevSegList& L) {
        buf(L.off);
        buf(L.pos);
        buf(L.a);
        buf(L.b);
        k.push_back(L.present ? 1 : 0);
      };
      buf(m->p);
      for (int a = 0; a < 3; ++a) {
        buf(m->coef[a]);
        buf(m->chunk[a]);
        buf(m->chunk_il[a]);
        buf(m->chunk_slots[a]);
      }
      for (const DevBuf* d : {&m->d_bulk_vox, &m->d_bulk_st, &m->d_bulk_su, &m->d_dir_vox,
                              &m->d_dir_val, &m->d_ag_vox_orig, &m->d_ag_t1, &m->d_ag_t2,
                              &m->d_ag_key, &m->d_ag_idx_in, &m->d_ag_idx, &m->d_sort_tmp,
                              &m->d_gather, &m->d_status})
        buf(*d);
      seg(m->seg_bulk);
      seg(m->seg_dir_x);
      seg(m->seg_dir_y);
      seg(m->seg_cells);
    }
  for (const GroupPlan& G : b->groups) k.append(reinterpret_cast<const char*>(&G), sizeof G);
  return k;
}

void batch_step(bfvm_batch* b, double dt, int nsteps, int flags) {
  require(nsteps >= 0, "negative step count");
  require((flags & ~BFVM_STEP_ALL) == 0, "unknown step flags");
  if (b->inst.empty() || nsteps == 0) return;
  prepare_instances(b, dt);
  plan(b, flags);
  const std::string key = plan_key(b, dt, nsteps, flags);
  if (!b->exec || key != b->key) {
    drop_graph(b);
    b->exec = capture(b, dt, nsteps, flags, 7, &b->graph_kernels);
    b->key = key;
  }
  BFVM_CUDA(cudaGraphLaunch(b->exec, b->stream));
  release_instances(b);
}

// Times `reps` replays of a graph of `steps` steps (or one axis's sweeps),
// returning the best milliseconds per replay.
float time_graph(bfvm_batch* b, double dt, int steps, int flags, int axes) {
  int64_t k = 0;
  cudaGraphExec_t exec = capture(b, dt, steps, flags, axes, &k);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float best = 1e30f;
  try {
    BFVM_CUDA(cudaEventCreate(&e0));
    BFVM_CUDA(cudaEventCreate(&e1));
    BFVM_CUDA(cudaGraphLaunch(exec, b->stream));  // warm-up
    for (int r = 0; r < 3; ++r) {
      BFVM_CUDA(cudaEventRecord(e0, b->stream));
      BFVM_CUDA(cudaGraphLaunch(exec, b->stream));
      BFVM_CUDA(cudaEventRecord(e1, b->stream));
      BFVM_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      BFVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      best = std::min(best, ms);
    }
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(exec);
  return best;
}

void batch_tune(bfvm_batch* b, double dt, int flags, int trial_steps) {
  require(trial_steps >= 1 && trial_steps <= 1000, "trial_steps must be in [1, 1000]");
  if (b->inst.empty()) return;
  prepare_instances(b, dt);
  // save the fields; the trial runs advance them
  size_t total = 0;
  for (bfvm_solver* m : b->inst) total += (m->NS() * m->elem() + 255) / 256 * 256;
  DevBuf save;
  save.ensure(std::max<size_t>(total, 16));
  auto copy_fields = [&](bool to_save) {
    size_t o = 0;
    for (bfvm_solver* m : b->inst) {
      const size_t bytes = m->NS() * m->elem();
      unsigned char* s = save.as<unsigned char>() + o;
      BFVM_CUDA(cudaMemcpyAsync(to_save ? s : m->p.ptr, to_save ? m->p.ptr : s, bytes,
                                cudaMemcpyDeviceToDevice, b->stream));
      o += (bytes + 255) / 256 * 256;
    }
  };
  copy_fields(true);
  const BatchConfig user = b->cfg;
  drop_graph(b);
  try {
    // 1. per axis: chunk length x threads, sweeps alone, default groups
    BatchConfig best = user;
    best.group_bytes = -1;
    for (int a = 0; a < 3; ++a) {
      float best_ms = 1e30f;
      for (int ch : {8, 16, 32})
        for (int th : {128, 256, 512}) {
          if (!config_fits(b, a, ch, th)) continue;
          b->cfg = best;
          b->cfg.mode = BFVM_BATCH_FUSED;  // the shapes are the fused kernels'
          b->cfg.ch[a] = ch;
          b->cfg.threads[a] = th;
          plan(b, BFVM_STEP_DIFFUSION);
          const float ms = time_graph(b, dt, trial_steps, BFVM_STEP_DIFFUSION, 1 << a);
          if (ms < best_ms) {
            best_ms = ms;
            best.ch[a] = ch;
            best.threads[a] = th;
          }
        }
    }
    // 2. every member's own sweep kernels and slabs (what branch mode runs;
    // each member's field is saved and restored by its tuner)
    for (bfvm_solver* m : b->inst) {
      BFVM_CUDA(cudaStreamSynchronize(b->stream));
      tune_sweeps(m, dt, 3);
    }
    // 3. the mode (and the persistent kernel's chunk length) and the group
    // budget, whole steps
    bool any_persistent = false, any_planes = false;
    for (const bfvm_solver* m : b->inst) {
      any_persistent = any_persistent || persistent_ok(m, 8);
      any_planes = any_planes || planes_ok(m);
    }
    float best_ms = 1e30f;
    int64_t best_budget = 0;
    int best_mode = BFVM_BATCH_FUSED, best_pch = best.pch;
    for (int mode :
         {BFVM_BATCH_FUSED, BFVM_BATCH_BRANCHES, BFVM_BATCH_PERSISTENT, BFVM_BATCH_PLANES}) {
      if (mode == BFVM_BATCH_PERSISTENT && (!any_persistent || !(flags & BFVM_STEP_DIFFUSION)))
        continue;
      if (mode == BFVM_BATCH_PLANES && (!any_planes || !(flags & BFVM_STEP_DIFFUSION) || !fp64(b)))
        continue;
      for (int pch : {8, 4, 16, 32, 0}) {
        if (pch != 8 && mode != BFVM_BATCH_PERSISTENT) continue;
        for (int64_t budget : {(int64_t)0, (int64_t)b->l2_bytes, (int64_t)b->l2_bytes / 2,
                               (int64_t)b->l2_bytes / 4, (int64_t)b->l2_bytes / 8}) {
          b->cfg = best;
          b->cfg.group_bytes = budget;
          b->cfg.mode = mode;
          b->cfg.pch = pch;
          plan(b, flags);
          const float ms = time_graph(b, dt, trial_steps, flags, 7);
          if (ms < best_ms) {
            best_ms = ms;
            best_budget = budget;
            best_mode = mode;
            best_pch = pch;
          }
        }
      }
    }
    best.group_bytes = best_budget;
    best.mode = best_mode;
    best.pch = best_pch;
    b->cfg = best;
  } catch (...) {
    b->cfg = user;
    copy_fields(false);
    cudaStreamSynchronize(b->stream);
    throw;
  }
  copy_fields(false);
  BFVM_CUDA(cudaStreamSynchronize(b->stream));
  release_instances(b);
}

#define BATCH_CALL(b, ...)                           \
  guarded([&] {                                      \
    require((b) != nullptr, "null batch handle");    \
    DeviceGuard dg_((b)->device);                    \
    __VA_ARGS__;                                     \
  })

}  // namespace
}  // namespace bfvm_rt

using namespace bfvm_rt;

extern "C" {

int bfvm_batch_create(bfvm_batch** out, int device) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    int ndev = 0;
    BFVM_CUDA(cudaGetDeviceCount(&ndev));
    require(device >= 0 && device < ndev, "no CUDA device " + std::to_string(device));
    DeviceGuard dg(device);
    bfvm_batch* b = new bfvm_batch;
    b->device = device;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) {
      if (b->stream) cudaStreamDestroy(b->stream);
      delete b;
      throw Error(BFVM_ERR_CUDA, "batch stream/event creation failed");
    }
    cudaDeviceGetAttribute(&b->l2_bytes, cudaDevAttrL2CacheSize, device);
    *out = b;
  });
}

int bfvm_batch_destroy(bfvm_batch* b) {
  if (!b) return BFVM_OK;
  return BATCH_CALL(b, {
    cudaStreamSynchronize(b->stream);
    drop_graph(b);
    b->d_desc.release();
    for (auto& sc : b->scratch) sc.buf.release();
    cudaEventDestroy(b->ev);
    cudaStreamDestroy(b->stream);
    delete b;
  });
}

int bfvm_batch_add(bfvm_batch* b, bfvm_solver* m) {
  return BATCH_CALL(b, {
    require(m != nullptr, "null solver handle");
    require(m->device == b->device, "instance lives on another device");
    require(m->precision != BFVM_FP32_FP64MATH,
            "batches take FP64 or FP32 instances (not BFVM_FP32_FP64MATH)");
    require(b->inst.empty() || m->precision == b->inst[0]->precision,
            "instances of one batch must share the precision");
    require(std::find(b->inst.begin(), b->inst.end(), m) == b->inst.end(),
            "instance already in the batch");
    b->inst.push_back(m);
  });
}

int bfvm_batch_clear(bfvm_batch* b) {
  return BATCH_CALL(b, {
    cudaStreamSynchronize(b->stream);
    b->inst.clear();
    for (auto& sc : b->scratch) sc.buf.release();
    b->scratch.clear();
    drop_graph(b);
  });
}

int bfvm_batch_size(bfvm_batch* b, int* count) {
  return BATCH_CALL(b, {
    require(count != nullptr, "null output pointer");
    *count = (int)b->inst.size();
  });
}

int bfvm_batch_step(bfvm_batch* b, double dt, int nsteps, int flags) {
  return BATCH_CALL(b, batch_step(b, dt, nsteps, flags));
}

int bfvm_batch_tune(bfvm_batch* b, double dt, int flags, int trial_steps) {
  return BATCH_CALL(b, batch_tune(b, dt, flags, trial_steps));
}

int bfvm_batch_set_config(bfvm_batch* b, const int* chunk, const int* threads,
                          int64_t group_bytes) {
  return BATCH_CALL(b, {
    require(group_bytes >= -1, "group_bytes must be -1 (default), 0 (one group) or positive");
    BatchConfig c;
    for (int a = 0; a < 3; ++a) {
      c.ch[a] = chunk ? chunk[a] : 0;
      c.threads[a] = threads ? threads[a] : 0;
      require(c.ch[a] == 0 || c.ch[a] == 8 || c.ch[a] == 16 || c.ch[a] == 32,
              "chunk must be 0, 8, 16 or 32");
      require(c.threads[a] == 0 || c.threads[a] == 128 || c.threads[a] == 256 ||
                  c.threads[a] == 512,
              "threads must be 0, 128, 256 or 512");
      require((c.ch[a] == 0) == (c.threads[a] == 0), "chunk and threads are set together");
    }
    c.group_bytes = group_bytes;
    c.mode = b->cfg.mode;
    c.pch = b->cfg.pch;
    b->cfg = c;
  });
}

int bfvm_batch_get_config(bfvm_batch* b, int* chunk, int* threads, int64_t* group_bytes) {
  return BATCH_CALL(b, {
    if (!b->inst.empty()) choose_shapes(b);
    for (int a = 0; a < 3; ++a) {
      if (chunk) chunk[a] = b->ch[a];
      if (threads) threads[a] = b->threads[a];
    }
    if (group_bytes)
      *group_bytes = b->cfg.group_bytes < 0 ? (int64_t)b->l2_bytes / 2 : b->cfg.group_bytes;
  });
}

int bfvm_batch_set_mode(bfvm_batch* b, int mode) {
  return BATCH_CALL(b, {
    require(mode == BFVM_BATCH_FUSED || mode == BFVM_BATCH_BRANCHES ||
                mode == BFVM_BATCH_PERSISTENT || mode == BFVM_BATCH_PLANES,
            "mode must be BFVM_BATCH_FUSED, BFVM_BATCH_BRANCHES, BFVM_BATCH_PERSISTENT or "
            "BFVM_BATCH_PLANES");
    b->cfg.mode = mode;
  });
}

int bfvm_batch_get_mode(bfvm_batch* b, int* mode) {
  return BATCH_CALL(b, {
    require(mode != nullptr, "null output pointer");
    *mode = b->cfg.mode;
  });
}

int bfvm_batch_set_persistent_chunk(bfvm_batch* b, int chunk) {
  return BATCH_CALL(b, {
    require(chunk == 0 || chunk == 4 || chunk == 8 || chunk == 16 || chunk == 32,
            "persistent chunk must be 4, 8, 16, 32 or 0 (whole lines)");
    b->cfg.pch = chunk;
  });
}

int bfvm_batch_get_persistent_chunk(bfvm_batch* b, int* chunk) {
  return BATCH_CALL(b, {
    require(chunk != nullptr, "null output pointer");
    *chunk = b->cfg.pch;
  });
}

int bfvm_batch_get_plan(bfvm_batch* b, int* groups, int64_t* kernels_per_call) {
  return BATCH_CALL(b, {
    if (groups) *groups = (int)b->groups.size();
    if (kernels_per_call) *kernels_per_call = b->exec ? b->graph_kernels : 0;
  });
}

int bfvm_batch_synchronize(bfvm_batch* b) {
  return BATCH_CALL(b, BFVM_CUDA(cudaStreamSynchronize(b->stream)));
}

}  // extern "C"
