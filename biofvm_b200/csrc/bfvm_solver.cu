// Host side of libbfvm.so: the C ABI of include/bfvm.h, the solver state
// (one BioFVM Microenvironment resident on one GPU) and the kernel launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "bfvm.h"
#include "bfvm_host_math.h"
#include "bfvm_kernels.cuh"
#include "bfvm_kernels_cluster.cuh"
#include "bfvm_kernels_grid.cuh"
#include "bfvm_kernels_tma.cuh"
#include <cub/device/device_radix_sort.cuh>
#include <cudaTypedefs.h>
#include <mutex>

#include "bfvm_state.h"

namespace bfvm_rt {

thread_local std::string g_last_error;

// Groups entries (already in non-decreasing (line, pos) order) by
// (line, chunk) segment.
std::vector<int> segment_offsets(int64_t nlines, int nchunks, int ch,
                                 const std::vector<int64_t>& line, const std::vector<int>& pos) {
  std::vector<int> off((size_t)(nlines * nchunks + 1), 0);
  for (size_t e = 0; e < line.size(); ++e) off[(size_t)(line[e] * nchunks + pos[e] / ch) + 1]++;
  for (size_t i = 1; i < off.size(); ++i) off[i] += off[i - 1];
  return off;
}

// Chunk length CH (points per thread) and block width TW (columns per block)
// per axis; a block is TW x NC threads with NC = ceil(n/CH) <= 512/TW.  The y
// and z sweeps of long lines take CH = 32 (fewer chunks to join per line).
// x takes the row kernel with CH = 32 where it was measured faster than the
// register kernel (S >= 4 densities and rows of >= 96 points: 0.85 -> 0.75 ms
// at 256^3 x 10 FP64, 4.4 -> 2.7 ms at 384^3 x 10, 0.66 -> 0.43 ms at
// 256^3 x 10 FP32), else the register kernel with CH = 8 or 16.
// Lines of up to this many points run in the chunked kernels (the chunks of a
// line in one block); longer lines run in long_line_kernel.
constexpr int kChunkedMaxN = 1024;
// most slabs of a z-split field
constexpr int kZSlabMaxRanks = 64;

bool long_axis(const bfvm_solver* m, int a) {
  return (a == 0 ? m->nx : (a == 1 ? m->ny : m->nz)) > kChunkedMaxN;
}

void choose_axes(bfvm_solver* m) {
  const int ns[3] = {m->nx, m->ny, m->nz};
  for (int a = 0; a < 3; ++a) {
    const int n = ns[a];
    if (m->axis[a].user && (n + m->axis[a].ch - 1) / m->axis[a].ch * m->axis[a].tw <=
                               bfvm::sweep_max_threads(m->axis[a].ch))
      continue;
    m->axis[a].user = false;
    m->axis[a].kind = 0;
    m->axis[a].stages = 0;
    int ch = (n <= 64) ? 8 : 16;
    if (a > 0 && n >= 128) ch = 32;
    while ((n + ch - 1) / ch > 16 && ch < 32) ch *= 2;
    const int nc = (n + ch - 1) / ch;
    // x: blocks of at most 256 threads (two per SM, measured faster at 256^3)
    const int maxt = (a == 0) ? std::min(256, bfvm::sweep_max_threads(ch))
                              : bfvm::sweep_max_threads(ch);
    int tw = 32;
    while (tw > 8 && nc * tw > maxt) tw /= 2;
    if (n > kChunkedMaxN) {  // the long-line kernel runs this axis
      m->axis[a].ch = 32;
      m->axis[a].tw = 1;
      continue;
    }
    require(nc * tw <= bfvm::sweep_max_threads(ch),
            "axis with " + std::to_string(n) + " points: no sweep kernel shape fits");
    m->axis[a].ch = ch;
    m->axis[a].tw = tw;
    if (a == 0 && m->S >= 4 && n >= 96 && (int64_t)m->S * ((n + 31) / 32) <= 256 &&
        ((int64_t)n * m->S * m->elem()) % 16 == 0) {
      m->axis[a].ch = 32;
      m->axis[a].kind = BFVM_PATH_TMA;
      tw = 32;
      while (tw > 8 && (n + 31) / 32 * tw > bfvm::sweep_max_threads(32)) tw /= 2;
      m->axis[a].tw = tw;
    }
  }
}

void clear_state_after_resize(bfvm_solver* m) {
  m->zs_ranks = 0;  // a z slab is declared again for the new mesh
  m->zs_bounds.clear();
  m->p.ensure(std::max<size_t>(m->NS() * m->elem(), 16));
  BFVM_CUDA(cudaMemsetAsync(m->p.ptr, 0, m->NS() * m->elem(), m->stream));
  m->setup_done = false;
  m->bulk_vox.clear();
  m->bulk_st.clear();
  m->bulk_su.clear();
  m->bulk_dirty = true;
  m->dir_vox.clear();
  m->dir_val.clear();
  m->dir_dirty = true;
  m->n_agents = 0;
  m->ag_dirty = m->ag_seg_dirty = true;
  m->d_grad.release();
  for (auto& A : m->axis) A.user = false;
  choose_axes(m);
}

// ---- Thomas coefficients ---------------------------------------------------

// The reference shares one set of Thomas coefficients between its 3-D and
// 2-D LOD solvers (diffusion_solver_setup_done): whichever runs first fixes
// them.
// z slab: the per-density constants that join the slabs of a z-split field
// (every slab's P = prod a, Gs, R = prod c over its planes) and this slab's
// per-plane G and Rk, from the global line's slopes a_k = c_k = -cx_k (the
// forward and backward slopes are the same numbers), in FP64.  With x' the
// slab-local solve (zero carries at both slab ends) and A_k the product of
// a over the slab's planes up to k:
//   G_k = A_k + c_k G_{k+1} (G past the slab 0), Rk_k = prod_{j>=k} c_j,
//   x_k = x'_k + C G_k + X Rk_k
// with C the true forward value before the slab and X the true solution on
// the first plane after it.
void zslab_tables(bfvm_solver* m, const std::vector<double>& gcx) {
  const int S = m->S, R = m->zs_ranks, ntot = m->zs_bounds[R];
  std::vector<double> cst((size_t)R * S * 3), pt((size_t)m->nz * S * 2);
  for (int r = 0; r < R; ++r) {
    const int g0 = m->zs_bounds[r], g1 = m->zs_bounds[r + 1];
    for (int s = 0; s < S; ++s) {
      auto a = [&](int k) { return -gcx[(size_t)k * S + s]; };
      auto c = [&](int k) { return k + 1 < ntot ? -gcx[(size_t)k * S + s] : 0.0; };
      std::vector<double> A(g1 - g0), G(g1 - g0 + 1, 0.0), Rk(g1 - g0 + 1, 1.0);
      double prod = 1.0;
      for (int k = g0; k < g1; ++k) A[k - g0] = prod = prod * a(k);
      for (int k = g1 - 1; k >= g0; --k) {
        G[k - g0] = A[k - g0] + c(k) * G[k - g0 + 1];
        Rk[k - g0] = c(k) * Rk[k - g0 + 1];
      }
      cst[((size_t)r * S + s) * 3 + 0] = prod;
      cst[((size_t)r * S + s) * 3 + 1] = G[0];
      cst[((size_t)r * S + s) * 3 + 2] = Rk[0];
      if (r == m->zs_rank)
        for (int k = g0; k < g1; ++k) {
          pt[((size_t)(k - g0) * S + s) * 2 + 0] = G[k - g0];
          pt[((size_t)(k - g0) * S + s) * 2 + 1] = Rk[k - g0];
        }
    }
  }
  upload(m->zs_const, cst, m->stream);
  upload(m->zs_pt, pt, m->stream);
}

void thomas_setup(bfvm_solver* m, double dt) {
  const int ns[3] = {m->nx, m->ny, m->nz};
  for (int a = 0; a < 3; ++a) {
    const int n = ns[a], S = m->S;
    std::vector<double> c1(S), den((size_t)n * S), cx((size_t)n * S);
    if (a == 2 && m->zs_ranks > 0) {
      // a z slab: the rows of the whole line's coefficients for its planes
      const int ntot = m->zs_bounds[m->zs_ranks], z0 = m->zs_bounds[m->zs_rank];
      std::vector<double> gden((size_t)ntot * S), gcx((size_t)ntot * S);
      bfvm::thomas_axis(ntot, S, m->dx, dt, m->D.data(), m->decay.data(), c1.data(),
                        gden.data(), gcx.data(), m->lod_dims);
      std::copy(gden.begin() + (size_t)z0 * S, gden.begin() + (size_t)(z0 + n) * S, den.begin());
      std::copy(gcx.begin() + (size_t)z0 * S, gcx.begin() + (size_t)(z0 + n) * S, cx.begin());
      zslab_tables(m, gcx);
    } else {
      // The reference uses mesh.dx for every axis (BioFVM_solvers.cpp:112-113).
      bfvm::thomas_axis(n, S, m->dx, dt, m->D.data(), m->decay.data(), c1.data(), den.data(),
                        cx.data(), m->lod_dims);
    }
    std::vector<double> tab((size_t)3 * n * S + S);
    for (size_t i = 0; i < (size_t)n * S; ++i) {
      const int s = (int)(i % S);
      tab[i] = 1.0 / den[i];
      tab[(size_t)n * S + i] = c1[s] / den[i];
      tab[(size_t)2 * n * S + i] = -cx[i];
    }
    for (int s = 0; s < S; ++s) tab[(size_t)3 * n * S + s] = c1[s];
    if (m->math_elem() == sizeof(double)) {
      upload(m->coef[a], tab, m->stream);
    } else {
      // FP32 arithmetic: roundings chosen along each line (error diffusion);
      // the chunk tables of the tile kernels follow the floats chosen for them
      const size_t nS = (size_t)n * S;
      std::vector<float> tf(3 * nS + S);
      std::vector<double> tden(nS), tcx(nS);
      bfvm::fp32_tables(n, S, c1.data(), den.data(), cx.data(), tf.data(), tf.data() + nS,
                        tf.data() + 2 * nS, tf.data() + 3 * nS, tden.data(), tcx.data());
      upload(m->coef[a], tf, m->stream);
      den.swap(tden);
      cx.swap(tcx);
    }
    m->h_c1[a] = c1;
    m->h_den[a] = den;
    m->h_cx[a] = cx;
    m->chunk_ch[a] = 0;
  }
  m->cl_tab_ok = false;
  m->setup_dt = dt;
  m->setup_D = m->D;
  m->setup_decay = m->decay;
  m->setup_done = true;
}

// Chunk tables of one axis for its current chunk length (rebuilt when the
// chunk length or the Thomas coefficients change).  Chunks whose tables are
// bit-identical share one slot: away from the two line ends the Thomas
// denominators converge to a fixed point, so most interior chunks of a long
// line are the same and the tables the kernels read stay small enough for L1.
//
// Two copies are kept (bfvm::ChunkCoef): the planar one, which the FP64 line
// kernel at 16-column tiles reads (its warps meet up to twenty distinct
// densities of two chunks, and the planar words cut its shared-memory
// wavefronts: y sweep 0.528 -> 0.486 ms at 256^3 x 10), and the interleaved
// one, which every other kernel reads (one 16-byte load per entry: faster in
// the row kernel, 0.656 against 0.828 ms, and in the half-width line tiles
// of 1024-point lines, whose warps meet at most eight densities).
template <typename T>
bfvm::ChunkCoef<T> chunk_view(bfvm_solver* m, int a, bool interleaved = false) {
  const int ns[3] = {m->nx, m->ny, m->nz};
  const int n = ns[a], S = m->S, ch = m->axis[a].ch;
  const int nc = (n + ch - 1) / ch;
  auto up4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  if (m->chunk_ch[a] != ch) {
    const size_t fk = (size_t)S * n * 2;
    std::vector<double> k1((size_t)nc * ch * S * 2, 0.0), kg((size_t)nc * ch * S * 2, 0.0),
        kc((size_t)nc * S * 4);
    bfvm::chunk_tables(n, S, ch, m->h_c1[a].data(), m->h_den[a].data(), m->h_cx[a].data(),
                       k1.data(), kg.data(), kc.data());
    (void)fk;
    // slot per chunk: the first earlier full-length chunk with identical tables
    const size_t cw = (size_t)ch * S * 2;  // elements of one chunk in k1 / kg
    std::vector<int> slot_of(nc);
    std::vector<int> slot_chunk;  // representative chunk of each slot
    for (int c = 0; c < nc; ++c) {
      const bool full = (c + 1) * ch <= n;
      int found = -1;
      if (full) {
        for (size_t sl = 0; sl < slot_chunk.size() && found < 0; ++sl) {
          const int r = slot_chunk[sl];
          if ((r + 1) * ch > n) continue;
          if (std::memcmp(&k1[r * cw], &k1[c * cw], cw * sizeof(double)) == 0 &&
              std::memcmp(&kg[r * cw], &kg[c * cw], cw * sizeof(double)) == 0 &&
              std::memcmp(&kc[(size_t)r * S * 4], &kc[(size_t)c * S * 4],
                          (size_t)S * 4 * sizeof(double)) == 0)
            found = (int)sl;
        }
      }
      if (found < 0) {
        found = (int)slot_chunk.size();
        slot_chunk.push_back(c);
      }
      slot_of[c] = found;
    }
    const size_t ns_ = slot_chunk.size();
    const size_t k1n = up4(ns_ * cw), kgn = up4(ns_ * cw), kcn = up4((size_t)nc * S * 4);
    std::vector<double> tab(k1n + kgn + kcn, 0.0), til(k1n + kgn + kcn, 0.0);
    // planar (tab): per point the S first components, then the S second
    // ones; per chunk the S values of each transfer constant in turn.
    // Interleaved (til): chunk_tables()'s own order.
    for (size_t sl = 0; sl < ns_; ++sl) {
      const size_t r = (size_t)slot_chunk[sl];
      std::copy_n(&k1[r * cw], cw, &til[sl * cw]);
      std::copy_n(&kg[r * cw], cw, &til[k1n + sl * cw]);
      for (size_t q = 0; q < (size_t)ch; ++q)
        for (size_t s = 0; s < (size_t)S; ++s)
          for (size_t j = 0; j < 2; ++j) {
            const size_t src = r * cw + (q * S + s) * 2 + j;
            const size_t dst = sl * cw + (q * 2 + j) * S + s;
            tab[dst] = k1[src];
            tab[k1n + dst] = kg[src];
          }
    }
    // transfer constants per chunk (not per slot): the fold reads every chunk
    std::copy_n(kc.data(), (size_t)nc * S * 4, &til[k1n + kgn]);
    for (size_t c = 0; c < (size_t)nc; ++c)
      for (size_t s = 0; s < (size_t)S; ++s)
        for (size_t j = 0; j < 4; ++j)
          tab[k1n + kgn + (c * 4 + j) * S + s] = kc[(c * S + s) * 4 + j];
    if (sizeof(T) == sizeof(double)) {
      upload(m->chunk[a], tab, m->stream);
      upload(m->chunk_il[a], til, m->stream);
    } else {
      std::vector<float> tf(tab.begin(), tab.end()), tfi(til.begin(), til.end());
      upload(m->chunk[a], tf, m->stream);
      upload(m->chunk_il[a], tfi, m->stream);
    }
    upload(m->chunk_slots[a], slot_of, m->stream);
    m->chunk_ch[a] = ch;
    m->chunk_nslots[a] = (int)ns_;
  }
  const size_t cw = (size_t)ch * S * 2;
  const size_t ns_ = (size_t)m->chunk_nslots[a];
  const size_t k1n = up4(ns_ * cw), kgn = up4(ns_ * cw);
  const T* base = (interleaved ? m->chunk_il[a] : m->chunk[a]).as<T>();
  bfvm::ChunkCoef<T> c;
  c.k1 = base;
  c.kg = base + k1n;
  c.kc = base + k1n + kgn;
  c.slot = m->chunk_slots[a].as<int>();
  c.ch = ch;
  c.nc = nc;
  c.tab_elems = (int)(k1n + kgn + up4((size_t)nc * S * 4));
  const T* vec_sections[3] = {c.k1, c.kg, c.kc};
  for (const T* q : vec_sections)
    require(reinterpret_cast<uintptr_t>(q) % (2 * sizeof(T)) == 0,
            "chunk table not aligned for vector loads", BFVM_ERR_STATE);
  return c;
}


// ---- host lists -> device ---------------------------------------------------

void build_bulk(bfvm_solver* m) {
  if (!m->bulk_dirty) return;
  ++m->lists_version;
  cudaStream_t st = m->stream;
  const int S = m->S;
  const int64_t E = (int64_t)m->bulk_vox.size();
  if (E == 0) {
    m->seg_bulk.present = false;
    m->bulk_dirty = false;
    return;
  }
  upload(m->d_bulk_vox, m->bulk_vox, st);
  upload(m->d_bulk_st, m->bulk_st, st);
  upload(m->d_bulk_su, m->bulk_su, st);
  // shared coefficient rows (bitwise-equal rows once): worth it when they
  // compress at least 4x and voxel indices fit int32
  m->bulk_rows = 0;
  if (m->N() < ((int64_t)1 << 31)) {
    std::unordered_map<std::string, int> seen;
    std::vector<int> vox32(E), row(E);
    std::vector<double> tab;
    const int64_t cap = std::max<int64_t>(1, E / 4);
    std::string key((size_t)S * 2 * sizeof(double), '\0');
    bool ok = true;
    for (int64_t e = 0; e < E && ok; ++e) {
      for (int s = 0; s < S; ++s) {
        std::memcpy(&key[(size_t)s * 2 * sizeof(double)], &m->bulk_st[e * S + s], sizeof(double));
        std::memcpy(&key[((size_t)s * 2 + 1) * sizeof(double)], &m->bulk_su[e * S + s],
                    sizeof(double));
      }
      auto it = seen.find(key);
      if (it == seen.end()) {
        if ((int64_t)seen.size() >= cap) {
          ok = false;
          break;
        }
        it = seen.emplace(key, (int)seen.size()).first;
        for (int s = 0; s < S; ++s) {
          tab.push_back(m->bulk_st[e * S + s]);
          tab.push_back(m->bulk_su[e * S + s]);
        }
      }
      row[e] = it->second;
      vox32[e] = (int)m->bulk_vox[e];
    }
    if (ok) {
      upload(m->d_bulk_vox32, vox32, st);
      upload(m->d_bulk_row, row, st);
      upload(m->d_bulk_tab, tab, st);
      m->bulk_rows = (int64_t)seen.size();
    }
  }
  const int ch = m->axis[0].ch, nc = (m->nx + ch - 1) / ch;
  std::vector<int64_t> line(E);
  std::vector<int> pos(E);
  for (int64_t e = 0; e < E; ++e) {
    line[e] = m->bulk_vox[e] / m->nx;
    pos[e] = (int)(m->bulk_vox[e] % m->nx);
  }
  std::vector<int> off = segment_offsets((int64_t)m->ny * m->nz, nc, ch, line, pos);
  upload(m->seg_bulk.off, off, st);
  upload(m->seg_bulk.pos, pos, st);
  upload(m->seg_bulk.a, m->bulk_st, st);
  upload(m->seg_bulk.b, m->bulk_su, st);
  m->seg_bulk.present = true;
  m->bulk_dirty = false;
  (void)S;
}

void build_dirichlet(bfvm_solver* m) {
  if (!m->dir_dirty) return;
  ++m->lists_version;
  cudaStream_t st = m->stream;
  const int S = m->S;
  // Nodes are applied in list order, so for a repeated voxel the last one
  // wins: keep the last occurrence only.
  std::unordered_map<int64_t, size_t> last;
  for (size_t d = 0; d < m->dir_vox.size(); ++d) last[m->dir_vox[d]] = d;
  std::vector<int64_t> vox;
  vox.reserve(last.size());
  for (auto& kv : last) vox.push_back(kv.first);
  std::sort(vox.begin(), vox.end());
  const int64_t E = (int64_t)vox.size();
  m->dir_unique = E;
  m->dir_sorted = vox;
  if (E == 0) {
    m->seg_dir_x.present = m->seg_dir_y.present = false;
    m->dir_dirty = false;
    return;
  }
  std::vector<double> val((size_t)E * S);
  for (int64_t e = 0; e < E; ++e)
    std::copy_n(&m->dir_val[last[vox[e]] * S], S, &val[(size_t)e * S]);
  upload(m->d_dir_vox, vox, st);
  upload(m->d_dir_val, val, st);

  // x sweep: lines are rows (k, j), points i
  {
    const int ch = m->axis[0].ch, nc = (m->nx + ch - 1) / ch;
    std::vector<int64_t> line(E);
    std::vector<int> pos(E);
    for (int64_t e = 0; e < E; ++e) {
      line[e] = vox[e] / m->nx;
      pos[e] = (int)(vox[e] % m->nx);
    }
    upload(m->seg_dir_x.off, segment_offsets((int64_t)m->ny * m->nz, nc, ch, line, pos), st);
    upload(m->seg_dir_x.pos, pos, st);
    upload(m->seg_dir_x.a, val, st);
    m->seg_dir_x.present = true;
  }
  // y sweep: lines are (k, i), points j
  {
    const int ch = m->axis[1].ch, nc = (m->ny + ch - 1) / ch;
    std::vector<int64_t> key(E);
    for (int64_t e = 0; e < E; ++e) {
      const int64_t v = vox[e];
      const int64_t i = v % m->nx, j = (v / m->nx) % m->ny, k = v / ((int64_t)m->nx * m->ny);
      key[e] = (k * m->nx + i) * m->ny + j;
    }
    std::vector<int64_t> order(E);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
    std::vector<int64_t> line(E);
    std::vector<int> pos(E);
    std::vector<double> vy((size_t)E * S);
    for (int64_t r = 0; r < E; ++r) {
      const int64_t e = order[r];
      line[r] = key[e] / m->ny;
      pos[r] = (int)(key[e] % m->ny);
      std::copy_n(&val[(size_t)e * S], S, &vy[(size_t)r * S]);
    }
    upload(m->seg_dir_y.off, segment_offsets((int64_t)m->nz * m->nx, nc, ch, line, pos), st);
    upload(m->seg_dir_y.pos, pos, st);
    upload(m->seg_dir_y.a, vy, st);
    m->seg_dir_y.present = true;
  }
  m->dir_dirty = false;
}

// Agents stably sorted by voxel on the device (radix sort of (voxel, list
// position) pairs; a radix sort is stable, so agents of one voxel keep their
// list order, BioFVM_microenvironment.cpp:626-633): keys[A] (voxels, checked
// to lie in [0, N)) into key/idx, on stream st.
void sort_agents(int64_t A, int64_t N, const uint64_t* keys_in, DevBuf& key, DevBuf& idx_in,
                 DevBuf& idx, DevBuf& tmp_buf, cudaStream_t st, bfvm_solver* m) {
  key.ensure(A * sizeof(uint64_t));
  idx_in.ensure(A * sizeof(int));
  idx.ensure(A * sizeof(int));
  bfvm::iota_kernel<<<(unsigned)blocks_for(A, 256), 256, 0, st>>>(idx_in.as<int>(), A);
  check_launch(m);
  int end_bit = 1;
  while (end_bit < 63 && ((int64_t)1 << end_bit) < N) ++end_bit;
  // as unsigned keys the (non-negative) voxel indices sort like the signed values
  size_t tmp = 0;
  BFVM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys_in, key.as<uint64_t>(),
                                            idx_in.as<int>(), idx.as<int>(), (int)A, 0, end_bit,
                                            st));
  tmp_buf.ensure(std::max<size_t>(tmp, 16));
  BFVM_CUDA(cub::DeviceRadixSort::SortPairs(tmp_buf.ptr, tmp, keys_in, key.as<uint64_t>(),
                                            idx_in.as<int>(), idx.as<int>(), (int)A, 0, end_bit,
                                            st));
}

void build_agents(bfvm_solver* m) {
  if (!m->ag_dirty) return;
  ++m->lists_version;
  const int64_t A = m->n_agents;
  m->ag_dirty = false;
  if (A == 0) return;
  sort_agents(A, m->N(), m->d_ag_vox_orig.as<uint64_t>(), m->d_ag_key, m->d_ag_idx_in,
              m->d_ag_idx, m->d_sort_tmp, m->stream, m);
}

// Segment lists of the agents for the fused x-sweep prologue: entries grouped
// by (x line, chunk), each group in sorted (voxel, list) order.  Built on the
// host from the device copy; only the fused-sources path uses them.
void build_agent_segments(bfvm_solver* m) {
  if (!m->ag_seg_dirty) return;
  const int S = m->S;
  const int64_t A = m->n_agents;
  m->ag_seg_dirty = false;
  if (A == 0) {
    m->seg_cells.present = false;
    return;
  }
  build_agents(m);
  cudaStream_t st = m->stream;
  std::vector<uint64_t> key(A);
  std::vector<int> idx(A);
  std::vector<double> t1_in((size_t)A * S), t2_in((size_t)A * S);
  BFVM_CUDA(cudaMemcpyAsync(key.data(), m->d_ag_key.ptr, A * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, st));
  BFVM_CUDA(cudaMemcpyAsync(idx.data(), m->d_ag_idx.ptr, A * sizeof(int), cudaMemcpyDeviceToHost,
                            st));
  BFVM_CUDA(cudaMemcpyAsync(t1_in.data(), m->d_ag_t1.ptr, t1_in.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  BFVM_CUDA(cudaMemcpyAsync(t2_in.data(), m->d_ag_t2.ptr, t2_in.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
  BFVM_CUDA(cudaStreamSynchronize(st));
  std::vector<int64_t> line(A);
  std::vector<int> pos(A);
  std::vector<double> t1((size_t)A * S), t2((size_t)A * S);
  for (int64_t r = 0; r < A; ++r) {
    const int64_t v = (int64_t)key[r], e = idx[r];
    line[r] = v / m->nx;
    pos[r] = (int)(v % m->nx);
    std::copy_n(&t1_in[(size_t)e * S], S, &t1[(size_t)r * S]);
    std::copy_n(&t2_in[(size_t)e * S], S, &t2[(size_t)r * S]);
  }
  const int ch = m->axis[0].ch, nc = (m->nx + ch - 1) / ch;
  upload(m->seg_cells.off, segment_offsets((int64_t)m->ny * m->nz, nc, ch, line, pos), st);
  upload(m->seg_cells.pos, pos, st);
  upload(m->seg_cells.a, t1, st);
  upload(m->seg_cells.b, t2, st);
  m->seg_cells.present = true;
}

// add_density on the agents: temp1/temp2 get one more column, 0 and 1 (the
// identity update) for the new density.
void widen_agents(bfvm_solver* m, int S0) {
  const int64_t A = m->n_agents;
  if (A == 0) return;
  const int S1 = S0 + 1;
  auto widen = [&](DevBuf& b, double fill) {
    DevBuf w;
    w.ensure((size_t)A * S1 * sizeof(double));
    BFVM_CUDA(cudaMemcpy2DAsync(w.ptr, S1 * sizeof(double), b.ptr, S0 * sizeof(double),
                                S0 * sizeof(double), A, cudaMemcpyDeviceToDevice, m->stream));
    bfvm::fill_column_kernel<<<(unsigned)blocks_for(A, 256), 256, 0, m->stream>>>(
        w.as<double>(), A, S1, S0, fill);
    check_launch(m);
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
    b.release();
    b = w;
    w.ptr = nullptr;
  };
  widen(m->d_ag_t1, 0.0);
  widen(m->d_ag_t2, 1.0);
}

void build_all(bfvm_solver* m) {
  build_bulk(m);
  build_dirichlet(m);
  build_agents(m);
  if (m->fuse_sources) build_agent_segments(m);
}

// ---- launches ---------------------------------------------------------------

template <typename T, typename CT, int CH, int MINB>
void launch_sweep_mb(const bfvm::SweepArgs<T, CT>& a, int mode, dim3 grid, dim3 block, size_t smem,
                     cudaStream_t st) {
  if (mode == bfvm::kSweepFull)
    bfvm::lod_sweep_kernel<T, CH, bfvm::kSweepFull, MINB, CT><<<grid, block, smem, st>>>(a);
  else if (mode == bfvm::kSweepDirEpi)
    bfvm::lod_sweep_kernel<T, CH, bfvm::kSweepDirEpi, MINB, CT><<<grid, block, smem, st>>>(a);
  else
    bfvm::lod_sweep_kernel<T, CH, bfvm::kSweepPlain, MINB, CT><<<grid, block, smem, st>>>(a);
}

template <typename T, typename CT, int CH>
void launch_sweep_ch(const bfvm::SweepArgs<T, CT>& a, int mode, int minb, dim3 grid, dim3 block,
                     size_t smem, cudaStream_t st) {
  if (minb == 2)
    launch_sweep_mb<T, CT, CH, 2>(a, mode, grid, block, smem, st);
  else
    launch_sweep_mb<T, CT, CH, 1>(a, mode, grid, block, smem, st);
}

// Sweeps take a range of z planes [z0, z1) for the x and y axes (z1 < 0:
// every plane): the x and y lines of a slab of planes are independent of the
// other planes' (see step_once).
template <typename T, typename CT>
void launch_sweep(bfvm_solver* m, int ax, int fuse, double dt, int64_t z0 = 0, int64_t z1 = -1) {
  const int S = m->S;
  const int64_t nx = m->nx, ny = m->ny, nz = m->nz;
  bfvm::SweepArgs<T, CT> a{};
  a.p = m->p.as<T>();
  a.out = m->sweep_out ? static_cast<T*>(m->sweep_out) : a.p;
  a.S = S;
  a.dt = dt;
  a.coef = coef_view<CT>(m, ax);
  const int64_t nzp = (m->lod_dims == 2) ? 1 : nz;  // planes swept
  if (ax == 0) {
    a.n = (int)nx;
    a.C = S;
    a.outer_stride = nx * S;
    a.line_stride = S;
    a.ncols = ny * nzp * S;
  } else if (ax == 1) {
    a.n = (int)ny;
    a.C = nx * S;
    a.outer_stride = nx * ny * S;
    a.line_stride = nx * S;
    a.ncols = nzp * nx * S;
  } else {
    a.n = (int)nz;
    a.C = nx * ny * S;
    a.outer_stride = 0;
    a.line_stride = nx * ny * S;
    a.ncols = nx * ny * S;
  }
  const Axis& A = m->axis[ax];
  a.nchunks = (a.n + A.ch - 1) / A.ch;
  if ((fuse & bfvm::kFuseBulk) && !m->seg_bulk.present) fuse &= ~bfvm::kFuseBulk;
  if ((fuse & bfvm::kFuseCells) && !m->seg_cells.present) fuse &= ~bfvm::kFuseCells;
  const DevSegList& dseg = (ax == 0) ? m->seg_dir_x : m->seg_dir_y;
  if (!dseg.present || ax == 2) fuse &= ~(bfvm::kFuseDirPro | bfvm::kFuseDirEpi);
  a.fuse = fuse;
  a.bulk = m->seg_bulk.view();
  a.cells = m->seg_cells.view();
  a.dir_pro = dseg.view();
  a.dir_epi = dseg.view();
  if (z1 >= 0 && ax < 2) {  // columns of planes z0 .. z1-1
    const int64_t per_plane = (ax == 0 ? ny : nx) * S;
    a.col0 = z0 * per_plane;
    a.ncols = z1 * per_plane;
  }
  // columns per block: the axis's choice, narrowed to the block size the
  // kernel is compiled for (a fallback from another kernel may bring a wider one)
  int tw = A.tw;
  while (tw > 1 && tw * a.nchunks > bfvm::sweep_max_threads(A.ch)) tw /= 2;
  require(tw * a.nchunks <= bfvm::sweep_max_threads(A.ch), "line too long for the sweep kernel",
          BFVM_ERR_STATE);
  dim3 block(tw, a.nchunks);
  dim3 grid((unsigned)blocks_for(a.ncols - a.col0, tw));
  const size_t smem = 4 * sizeof(CT) * (size_t)tw * a.nchunks;
  int mode = bfvm::kSweepPlain;
  if (fuse & (bfvm::kFuseBulk | bfvm::kFuseCells | bfvm::kFuseDirPro))
    mode = bfvm::kSweepFull;
  else if (fuse & bfvm::kFuseDirEpi)
    mode = bfvm::kSweepDirEpi;
  switch (A.ch) {
    case 8: launch_sweep_ch<T, CT, 8>(a, mode, A.minb, grid, block, smem, m->stream); break;
    case 16: launch_sweep_ch<T, CT, 16>(a, mode, A.minb, grid, block, smem, m->stream); break;
    case 32: launch_sweep_ch<T, CT, 32>(a, mode, A.minb, grid, block, smem, m->stream); break;
    default: throw Error(BFVM_ERR_STATE, "unsupported chunk length");
  }
  check_launch(m);
}

// ---- TMA-fed persistent sweeps ---------------------------------------------

// The driver's tensor-map encoder, looked up once (a static initialised by
// the first caller; other threads wait for it; a failed lookup is retried).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    BFVM_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
    require(q == cudaDriverEntryPointSuccess && ptr != nullptr,
            "cuTensorMapEncodeTiled is not available from the driver", BFVM_ERR_CUDA);
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }();
  return fn;
}

// Raises the dynamic shared-memory limit of a kernel once per device (solvers
// on other host threads may launch the same kernels: the record is locked).
void allow_smem(const void* kernel, int device, size_t bytes) {
  static std::mutex mu;
  static std::unordered_map<const void*, uint64_t> done;  // kernel -> device bitmask
  require(device >= 0 && device < 64, "device index out of range");
  std::lock_guard<std::mutex> g(mu);
  uint64_t& mask = done[kernel];
  if (mask & (1ull << device)) return;
  // a block may have 227 KB in all: the kernel's static shared memory counts
  cudaFuncAttributes fa;
  BFVM_CUDA(cudaFuncGetAttributes(&fa, kernel));
  const int limit = 227 * 1024 - (int)fa.sharedSizeBytes;
  require(bytes <= (size_t)limit, "kernel needs more shared memory than a block may have",
          BFVM_ERR_STATE);
  BFVM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
  mask |= 1ull << device;
}

constexpr size_t kSmemBudget = 224 * 1024;  // of the 227 KB a block may use

// Shared-memory bytes of an axis's chunk tables plus slot map (for staging
// them per block); 0 if the tables are not built yet.
size_t table_bytes(const bfvm_solver* m, int a) {
  if (m->chunk_ch[a] != m->axis[a].ch || m->chunk_nslots[a] == 0) return 0;
  auto up4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
  const int ns[3] = {m->nx, m->ny, m->nz};
  const size_t ch = m->axis[a].ch, S = m->S, nsl = m->chunk_nslots[a];
  const size_t nc = (ns[a] + ch - 1) / ch;
  const size_t elems = up4(nsl * ch * S * 2) * 2 + up4(nc * S * 4);
  return elems * m->math_elem() + nc * sizeof(int) + 16;
}

struct LinesPlan {
  bool ok = false;
  bool smem_tab = false;
  int n = 0, ch = 0, nc = 0, w = 0, stages = 0, box_n = 0, nboxes = 0;
  int64_t C = 0, nouter = 0, ls = 0, os = 0;
  size_t smem = 0;
};

// y (ax = 1) or z (ax = 2) sweep as a 3-D tensor [outer][n][C].  Tiles are
// 16 columns wide in FP64 and 32 in FP32 (128-byte rows), half that for lines
// of 17-32 chunks; the ring gets as many stages as keep two blocks per SM,
// else one block with more stages.
LinesPlan plan_lines(const bfvm_solver* m, int ax) {
  LinesPlan L;
  const int64_t es = (int64_t)m->elem();
  const int64_t nx = m->nx, ny = m->ny, nz = m->nz, S = m->S;
  if (ax == 0) {
    // x lines: the densities of a voxel are the columns, the rows the outer
    // blocks (rows too long for the row kernel's tiles)
    L.n = (int)nx; L.C = S; L.nouter = ny * ((m->lod_dims == 2) ? 1 : nz); L.ls = S;
    L.os = nx * S;
  } else if (ax == 1) {
    L.n = (int)ny; L.C = nx * S; L.nouter = (m->lod_dims == 2) ? 1 : nz; L.ls = nx * S;
    L.os = nx * ny * S;
  } else {
    L.n = (int)nz; L.C = nx * ny * S; L.nouter = 1; L.ls = nx * ny * S; L.os = nx * ny * nz * S;
  }
  if ((L.ls * es) % 16 || (L.os * es) % 16 || L.n > 1024 || L.C >= ((int64_t)1 << 31)) return L;
  // the chunk length of the axis: the (line, chunk) segment lists are built with it
  L.ch = m->axis[ax].ch;
  L.nc = (L.n + L.ch - 1) / L.ch;
  L.w = (m->math_elem() == 8) ? 16 : 32;
  if (L.nc > 32 || (L.nc > 16 && L.ch < 32)) return L;
  if (L.nc > 16) L.w /= 2;  // 513-1024 points: half-width tiles, 32 chunks
  if (ax == 0 && L.C % L.w) return L;  // x: whole tiles of densities only
  L.box_n = std::min(L.n, 256);
  L.nboxes = (L.n + L.box_n - 1) / L.box_n;
  const int64_t ctiles = (L.C + L.w - 1) / L.w;
  if (ctiles * L.nouter >= ((int64_t)1 << 31)) return L;
  const size_t stage = (size_t)L.box_n * L.nboxes * L.w * es;
  const size_t fold = 4 * (size_t)L.nc * L.w * m->math_elem();  // two parities of (qe, x0) pairs
  const size_t extra = 8 * 4 + 128;
  const size_t tab = table_bytes(m, ax);
  // preferred: the chunk tables staged in shared memory, two blocks per SM
  // (about 113 KB each); else one block; else tables read through L1.
  auto stages_for = [&](size_t budget, size_t t) -> int {
    return budget > fold + extra + t ? (int)std::min<size_t>(4, (budget - fold - extra - t) / stage)
                                     : 0;
  };
  L.smem_tab = tab > 0;
  L.stages = L.smem_tab ? stages_for(113 * 1024, tab) : 0;
  if (L.stages < 2 && L.smem_tab) L.stages = stages_for(kSmemBudget, tab);
  if (L.stages < 2) {
    L.smem_tab = false;
    L.stages = stages_for(80 * 1024, 0);
    if (L.stages < 2) L.stages = stages_for(kSmemBudget, 0);
    if (L.stages < 2) return L;
  }
  // tuning overrides for measurements: BFVM_LINES_TAB=0|1 (tables in shared
  // memory), BFVM_LINES_STAGES=2..4 (ring depth; shared memory permitting)
  static const char* env_tab = std::getenv("BFVM_LINES_TAB");
  static const char* env_st = std::getenv("BFVM_LINES_STAGES");
  if (env_tab || env_st) {
    const bool want_tab = env_tab ? std::atoi(env_tab) != 0 && tab > 0 : L.smem_tab;
    const int want_st = env_st ? std::max(2, std::min(4, std::atoi(env_st))) : L.stages;
    if (stages_for(kSmemBudget, want_tab ? tab : 0) >= want_st) {
      L.smem_tab = want_tab;
      L.stages = want_st;
    }
  }
  L.smem = L.stages * stage + fold + extra + (L.smem_tab ? tab : 0);
  L.ok = true;
  return L;
}

// Density counts the row kernel has builds for (bfvm_set_row_build).
bool row_build_count(int S) { return S == 4 || S == 8 || S == 10 || S == 16; }

struct RowsPlan {
  bool ok = false;
  bool smem_tab = false;
  int build = 0;  // row build that runs (Axis::build where it applies, else 0)
  int ch = 0, nc = 0, R = 0, stages = 0, maxt = 256;
  int tpc = 0;  // threads per chunk
  int minb = 1;  // resident blocks per SM the kernel is compiled for
  int64_t pitch = 0;
  size_t smem = 0;
};

// x sweep: tiles of R whole rows, one block per SM of R*S*NC <= 512 threads.
// Rows sit in shared memory at a padded pitch (16-byte multiple, = S modulo
// 16 elements where possible) so the column-major thread mapping is free of
// bank conflicts.
RowsPlan plan_rows(const bfvm_solver* m) {
  RowsPlan P;
  const int64_t es = (int64_t)m->elem();
  const int64_t row_elems = (int64_t)m->nx * m->S;
  const int64_t row_bytes = row_elems * es;
  const int64_t rows = (int64_t)m->ny * (m->lod_dims == 2 ? 1 : m->nz);
  if (row_bytes % 16 || m->nx > 1024) return P;
  P.ch = m->axis[0].ch;
  P.nc = (m->nx + P.ch - 1) / P.ch;
  const int cols = m->S * P.nc;  // threads of one row
  if (cols <= 0 || cols > 512) return P;
  // pitch: row_elems rounded up so that pitch == S (mod 16 elements of 8 B,
  // 32 of 4 B) and pitch*es is a multiple of 16 bytes
  const int64_t mod = (es == 8) ? 16 : 32, step = 16 / es;
  int64_t pitch = row_elems;
  for (int64_t k = 0; k < mod; k += step) {
    if (((row_elems + k) - m->S) % mod == 0) {
      pitch = row_elems + k;
      break;
    }
  }
  if (pitch == row_elems && (row_elems - m->S) % mod != 0)
    pitch = (row_elems + step - 1) / step * step;
  P.pitch = pitch;
  const size_t extra = 8 * 4 + 16 + 128;
  const size_t tab = table_bytes(m, 0);
  // tiles in the ring: 2, or 3 (one more tile in flight while a tile is
  // solved) where the axis asks for it
  const int nst = m->axis[0].stages == 3 ? 3 : 2;
  // Blocks of at most 256 threads (room for each thread's chunk in
  // registers), a 2-stage ring of R rows, the chunk tables in shared memory
  // when they fit; else one block of up to 512 threads.  Half the shared
  // memory per block where the kernel is compiled for two blocks per SM
  // (chunks of up to 16 points), all of it where one block fills the
  // register file (32-point chunks).
  for (int maxt : {256, 512}) {
    if (cols > maxt) continue;
    // two blocks per SM also at 32-point chunks where the axis asks for it
    const int minb = (maxt == 256 && P.ch == 32 && m->axis[0].minb == 2)
                         ? 2
                         : bfvm::rows_min_blocks(P.ch, maxt);
    const size_t budget = minb == 2 ? 113 * 1024 : kSmemBudget;
    for (int staged = 1; staged >= 0; --staged) {
      if (staged && tab == 0) continue;
      for (int R = (int)std::min<int64_t>(maxt / cols, rows); R >= 1; --R) {
        const size_t stage = (size_t)(R * pitch * es);
        const size_t fold = 4 * (size_t)P.nc * R * m->S * m->math_elem();  // two parities of (qe, x0)
        const size_t t = staged ? tab : 0;
        const size_t smem = nst * stage + fold + extra + t;
        if (smem > budget) continue;
        P.R = R;
        // whole warps per chunk when that still fits the block: the lanes
        // of a warp then read one chunk (two chunks' rows would share banks)
        const int fw = R * m->S, fw32 = (fw + 31) / 32 * 32;
        P.tpc = fw32 * P.nc <= maxt ? fw32 : fw;
        P.stages = nst;
        P.minb = minb;
        P.maxt = maxt;
        P.smem_tab = staged != 0;
        P.smem = smem;
        P.ok = true;
        // the builds for one density count exist for FP64 rows at 32-point
        // chunks, tables in shared memory, one block of <= 256 threads per
        // SM and a two-tile ring, with 4, 8, 10 or 16 densities
        const int b = m->axis[0].build;
        P.build = (b != 0 && es == 8 && m->math_elem() == 8 && P.ch == 32 && P.smem_tab &&
                   maxt == 256 && minb == 1 && nst == 2 && row_build_count(m->S))
                      ? b
                      : 0;
        return P;
      }
    }
  }
  return P;
}

template <typename T, typename CT, int CH, int ST, bool DIR, bool TAB, int MAXNC, int W>
void launch_lines_nc(const CUtensorMap& map, const bfvm::LinesArgs<T, CT>& a, int ntiles,
                     dim3 block, size_t smem, bfvm_solver* m) {
  require((int)block.x == W && (int)block.y <= MAXNC, "line kernel launch shape",
          BFVM_ERR_STATE);
  auto k = bfvm::lod_lines_tma_kernel<T, CH, W, ST, DIR, TAB, MAXNC, CT>;
  allow_smem((const void*)k, m->device, smem);
  int per_sm = 0;
  BFVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block.x * block.y, smem));
  require(per_sm > 0, "sweep kernel does not fit on an SM", BFVM_ERR_STATE);
  dim3 grid((unsigned)std::min<int64_t>(ntiles, (int64_t)per_sm * m->num_sms));
  k<<<grid, block, smem, m->stream>>>(map, a);
}

// Lines of up to 8 chunks of 32 points take the kernel compiled for 8 chunks
// (more registers per thread); up to 16 chunks the one for 16; lines of 17 to
// 32 chunks of 32 points (513-1024 points) the one for 32 chunks with tiles of
// half the width (the same threads per block and registers per thread).
template <typename T, typename CT, int CH, int ST, bool DIR, bool TAB>
void launch_lines_inst(const CUtensorMap& map, const bfvm::LinesArgs<T, CT>& a, int ntiles,
                       dim3 block, size_t smem, bfvm_solver* m) {
  constexpr int WF = sizeof(CT) == 8 ? 16 : 32;  // 128-byte tile rows
  if constexpr (CH >= 32) {
    if (block.y > 16) {
      launch_lines_nc<T, CT, CH, ST, DIR, TAB, 32, WF / 2>(map, a, ntiles, block, smem, m);
      return;
    }
    if (block.y <= 8) {
      launch_lines_nc<T, CT, CH, ST, DIR, TAB, 8, WF>(map, a, ntiles, block, smem, m);
      return;
    }
  }
  launch_lines_nc<T, CT, CH, ST, DIR, TAB, 16, WF>(map, a, ntiles, block, smem, m);
}

template <typename T, typename CT, int CH, int ST, bool TAB>
void launch_lines_dir(const CUtensorMap& map, const bfvm::LinesArgs<T, CT>& a, bool dir, int ntiles,
                      dim3 block, size_t smem, bfvm_solver* m) {
  if (dir)
    launch_lines_inst<T, CT, CH, ST, true, TAB>(map, a, ntiles, block, smem, m);
  else
    launch_lines_inst<T, CT, CH, ST, false, TAB>(map, a, ntiles, block, smem, m);
}

template <typename T, typename CT, int CH, int ST>
void launch_lines_tab(const CUtensorMap& map, const bfvm::LinesArgs<T, CT>& a, bool dir, bool tab,
                      int ntiles, dim3 block, size_t smem, bfvm_solver* m) {
  if (tab)
    launch_lines_dir<T, CT, CH, ST, true>(map, a, dir, ntiles, block, smem, m);
  else
    launch_lines_dir<T, CT, CH, ST, false>(map, a, dir, ntiles, block, smem, m);
}

template <typename T, typename CT, int CH>
void launch_lines_st(const CUtensorMap& map, const bfvm::LinesArgs<T, CT>& a, int stages, bool dir,
                     bool tab, int ntiles, dim3 block, size_t smem, bfvm_solver* m) {
  switch (stages) {
    case 2: launch_lines_tab<T, CT, CH, 2>(map, a, dir, tab, ntiles, block, smem, m); break;
    case 3: launch_lines_tab<T, CT, CH, 3>(map, a, dir, tab, ntiles, block, smem, m); break;
    default: launch_lines_tab<T, CT, CH, 4>(map, a, dir, tab, ntiles, block, smem, m); break;
  }
}

template <typename T, typename CT>
void launch_lines(bfvm_solver* m, int ax, const LinesPlan& L, bool dir, int64_t z0 = 0,
                  int64_t z1 = -1) {
  // (re)encode the tensor map when the field or its geometry changed
  const int64_t es = (int64_t)sizeof(T);
  const int64_t geom[9] = {(int64_t)(uintptr_t)m->p.ptr, es, L.C, L.n, L.nouter, L.ls, L.os,
                           L.w, L.box_n};
  if (!std::equal(geom, geom + 9, m->map_geom[ax])) {
    cuuint64_t dims[3] = {(cuuint64_t)L.C, (cuuint64_t)L.n, (cuuint64_t)L.nouter};
    cuuint64_t strides[2] = {(cuuint64_t)(L.ls * es), (cuuint64_t)(L.os * es)};
    cuuint32_t box[3] = {(cuuint32_t)L.w, (cuuint32_t)L.box_n, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = tensor_map_encoder()(
        &m->maps[ax], sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
        3, m->p.ptr, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    require(r == CUDA_SUCCESS, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")",
            BFVM_ERR_CUDA);
    std::copy(geom, geom + 9, m->map_geom[ax]);
  }
  bfvm::LinesArgs<T, CT> a{};
  a.p = m->p.as<T>();
  a.out = m->sweep_out ? static_cast<T*>(m->sweep_out) : a.p;
  a.C = L.C;
  a.n = L.n;
  a.ls = L.ls;
  a.os = L.os;
  a.S = m->S;
  a.ctiles = (uint32_t)((L.C + L.w - 1) / L.w);
  a.ntiles = (uint32_t)(a.ctiles * L.nouter);
  if (z1 >= 0 && ax == 1) {  // the outer blocks of the y lines are the z planes
    a.tile0 = (uint32_t)(a.ctiles * z0);
    a.ntiles = (uint32_t)(a.ctiles * z1);
  } else if (z1 >= 0 && ax == 0) {  // those of the x lines the rows, ny per plane
    a.tile0 = (uint32_t)(a.ctiles * z0 * m->ny);
    a.ntiles = (uint32_t)(a.ctiles * z1 * m->ny);
  }
  const int run_tiles = (int)(a.ntiles - a.tile0);
  a.box_n = L.box_n;
  a.nboxes = L.nboxes;
  a.nchunks = L.nc;
  a.cc = chunk_view<CT>(m, ax, /*interleaved=*/!bfvm::lines_planar((int)sizeof(CT), L.w));
  a.status = m->d_status.as<int>();
  if (dir) a.dir_epi = m->seg_dir_y.view();
  dim3 block(L.w, L.nc);
  switch (L.ch) {
    case 8: launch_lines_st<T, CT, 8>(m->maps[ax], a, L.stages, dir, L.smem_tab, run_tiles, block, L.smem, m); break;
    case 16: launch_lines_st<T, CT, 16>(m->maps[ax], a, L.stages, dir, L.smem_tab, run_tiles, block, L.smem, m); break;
    default: launch_lines_st<T, CT, 32>(m->maps[ax], a, L.stages, dir, L.smem_tab, run_tiles, block, L.smem, m); break;
  }
  check_launch(m);
}

template <typename T, typename CT, int CH, int MODE>
void launch_direct_inst(const bfvm::DirectArgs<T, CT>& a, dim3 grid, dim3 block, bfvm_solver* m) {
  constexpr int W = 32;
  auto k = bfvm::lod_sweep_direct_kernel<T, CH, W, MODE, CT>;
  // fold pairs + per-chunk constants + slot map
  const size_t smem = sizeof(CT) * 2 * block.x * block.y + sizeof(CT) * 4 * block.y * a.S +
                      sizeof(int) * block.y + 16;
  k<<<grid, block, smem, m->stream>>>(a);
}

template <typename T, typename CT, int CH>
void launch_direct_mode(const bfvm::DirectArgs<T, CT>& a, int mode, dim3 grid, dim3 block,
                        bfvm_solver* m) {
  if (mode == bfvm::kSweepFull)
    launch_direct_inst<T, CT, CH, bfvm::kSweepFull>(a, grid, block, m);
  else if (mode == bfvm::kSweepDirEpi)
    launch_direct_inst<T, CT, CH, bfvm::kSweepDirEpi>(a, grid, block, m);
  else
    launch_direct_inst<T, CT, CH, bfvm::kSweepPlain>(a, grid, block, m);
}

// Any axis with direct loads: blocks of 32 columns x all chunks of a line.
template <typename T, typename CT>
bool launch_direct(bfvm_solver* m, int ax, int fuse, double dt, int64_t z0 = 0,
                   int64_t z1 = -1) {
  const int64_t nx = m->nx, ny = m->ny, nz = m->nz, S = m->S;
  bfvm::DirectArgs<T, CT> a{};
  const int64_t nzp = (m->lod_dims == 2) ? 1 : nz;  // planes swept
  if (ax == 0) {
    a.n = (int)nx; a.C = S; a.outer_stride = nx * S; a.line_stride = S; a.ncols = ny * nzp * S;
  } else if (ax == 1) {
    a.n = (int)ny; a.C = nx * S; a.outer_stride = nx * ny * S; a.line_stride = nx * S;
    a.ncols = nzp * nx * S;
  } else {
    a.n = (int)nz; a.C = nx * ny * S; a.outer_stride = 0; a.line_stride = nx * ny * S;
    a.ncols = nx * ny * S;
  }
  if (z1 >= 0 && ax < 2) {  // columns of planes z0 .. z1-1
    const int64_t per_plane = (ax == 0 ? ny : nx) * S;
    a.col0 = z0 * per_plane;
    a.ncols = z1 * per_plane;
  }
  const int ch = m->axis[ax].ch;
  const int nc = (a.n + ch - 1) / ch;
  constexpr int W = 32;
  const int64_t nblocks = (a.ncols - a.col0 + W - 1) / W;
  if (W * nc > 512 || nblocks >= ((int64_t)1 << 31)) return false;
  a.p = m->p.as<T>();
  a.out = m->sweep_out ? static_cast<T*>(m->sweep_out) : a.p;
  a.S = (int)S;
  a.nchunks = nc;
  a.cc = chunk_view<CT>(m, ax, /*interleaved=*/true);
  a.dt = dt;
  if ((fuse & bfvm::kFuseBulk) && !m->seg_bulk.present) fuse &= ~bfvm::kFuseBulk;
  if ((fuse & bfvm::kFuseCells) && !m->seg_cells.present) fuse &= ~bfvm::kFuseCells;
  const DevSegList& dseg = (ax == 0) ? m->seg_dir_x : m->seg_dir_y;
  if (!dseg.present || ax == 2) fuse &= ~(bfvm::kFuseDirPro | bfvm::kFuseDirEpi);
  a.fuse = fuse;
  a.bulk = m->seg_bulk.view();
  a.cells = m->seg_cells.view();
  a.dir_pro = dseg.view();
  a.dir_epi = dseg.view();
  int mode = bfvm::kSweepPlain;
  if (fuse & (bfvm::kFuseBulk | bfvm::kFuseCells | bfvm::kFuseDirPro))
    mode = bfvm::kSweepFull;
  else if (fuse & bfvm::kFuseDirEpi)
    mode = bfvm::kSweepDirEpi;
  dim3 block(W, nc);
  dim3 grid((unsigned)nblocks);
  switch (ch) {
    case 8: launch_direct_mode<T, CT, 8>(a, mode, grid, block, m); break;
    case 16: launch_direct_mode<T, CT, 16>(a, mode, grid, block, m); break;
    default: launch_direct_mode<T, CT, 32>(a, mode, grid, block, m); break;
  }
  check_launch(m);
  return true;
}

template <typename T, typename CT, int CH, bool TAB, int MAXT, int ST,
          int MINB = bfvm::rows_min_blocks(CH, MAXT)>
void launch_rows_inst(const bfvm::RowsArgs<T, CT>& a, dim3 block, size_t smem, bfvm_solver* m,
                      int build = 0) {
  auto k = bfvm::lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB>;
  if constexpr (std::is_same<T, double>::value && std::is_same<CT, double>::value && CH == 32 &&
                TAB && MAXT == 256 && ST == 2 && MINB == 1) {
    if (build != 0) {
      require(row_build_count(a.S), "row build for another density count", BFVM_ERR_STATE);
      const bool pl = build == 2;
      using bfvm::lod_rows_tma_kernel;
      switch (a.S) {
        case 4:
          k = pl ? lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 4, true>
                 : lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 4, false>;
          break;
        case 8:
          k = pl ? lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 8, true>
                 : lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 8, false>;
          break;
        case 10:
          k = pl ? lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 10, true>
                 : lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 10, false>;
          break;
        default:
          k = pl ? lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 16, true>
                 : lod_rows_tma_kernel<T, CH, ST, TAB, MAXT, CT, MINB, 16, false>;
          break;
      }
    }
  } else {
    require(build == 0, "row build without a kernel", BFVM_ERR_STATE);
  }
  allow_smem((const void*)k, m->device, smem);
  int per_sm = 0;
  BFVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, block.x * block.y, smem));
  require(per_sm > 0, "sweep kernel does not fit on an SM", BFVM_ERR_STATE);
  dim3 grid((unsigned)std::min<int64_t>(a.ntiles - a.tile0, (int64_t)per_sm * m->num_sms));
  k<<<grid, block, smem, m->stream>>>(a);
}

template <typename T, typename CT, int CH, int ST>
void launch_rows_st(const bfvm::RowsArgs<T, CT>& a, const RowsPlan& P, dim3 block, bfvm_solver* m) {
  if (P.maxt == 256 && CH == 32 && P.minb == 2) {
    if (P.smem_tab)
      launch_rows_inst<T, CT, CH, true, 256, ST, 2>(a, block, P.smem, m);
    else
      launch_rows_inst<T, CT, CH, false, 256, ST, 2>(a, block, P.smem, m);
  } else if (P.maxt == 256) {
    if (P.smem_tab)
      launch_rows_inst<T, CT, CH, true, 256, ST>(a, block, P.smem, m, P.build);
    else
      launch_rows_inst<T, CT, CH, false, 256, ST>(a, block, P.smem, m);
  } else {
    if (P.smem_tab)
      launch_rows_inst<T, CT, CH, true, 512, ST>(a, block, P.smem, m);
    else
      launch_rows_inst<T, CT, CH, false, 512, ST>(a, block, P.smem, m);
  }
}

template <typename T, typename CT, int CH>
void launch_rows_ch(const bfvm::RowsArgs<T, CT>& a, const RowsPlan& P, dim3 block, bfvm_solver* m) {
  if (P.stages == 3)
    launch_rows_st<T, CT, CH, 3>(a, P, block, m);
  else
    launch_rows_st<T, CT, CH, 2>(a, P, block, m);
}

template <typename T, typename CT>
void launch_rows(bfvm_solver* m, const RowsPlan& P, int fuse, double dt, int64_t z0 = 0,
                 int64_t z1 = -1) {
  bfvm::RowsArgs<T, CT> a{};
  a.p = m->p.as<T>();
  a.out = m->sweep_out ? static_cast<T*>(m->sweep_out) : a.p;
  a.rows = (int64_t)m->ny * (m->lod_dims == 2 ? 1 : m->nz);
  a.n = m->nx;
  a.S = m->S;
  a.ntiles = (a.rows + P.R - 1) / P.R;
  if (z1 >= 0) {
    // tiles of R rows from the first one starting in plane z0 to the last
    // one starting before plane z1: a slab's rows that begin in an earlier
    // tile were swept with the slab before
    const int64_t r0 = z0 * m->ny, r1 = z1 * m->ny;
    a.tile0 = (r0 + P.R - 1) / P.R;
    a.ntiles = std::min(a.ntiles, (r1 + P.R - 1) / P.R);
    if (a.ntiles <= a.tile0) return;  // every row of the slab was swept before
  }
  a.nchunks = P.nc;
  a.R = P.R;
  a.pitch = P.pitch;
  a.cc = chunk_view<CT>(m, 0, /*interleaved=*/P.build != 2);
  a.dt = dt;
  if ((fuse & bfvm::kFuseBulk) && !m->seg_bulk.present) fuse &= ~bfvm::kFuseBulk;
  if ((fuse & bfvm::kFuseCells) && !m->seg_cells.present) fuse &= ~bfvm::kFuseCells;
  if (!m->seg_dir_x.present) fuse &= ~(bfvm::kFuseDirPro | bfvm::kFuseDirEpi);
  a.fuse = fuse;
  a.bulk = m->seg_bulk.view();
  a.cells = m->seg_cells.view();
  a.dir = m->seg_dir_x.view();
  a.status = m->d_status.as<int>();
  a.tpc = P.tpc;
  // whole warps: threads past tpc*NC idle through the sweep
  dim3 block((unsigned)((P.tpc * P.nc + 31) / 32 * 32));
  switch (P.ch) {
    case 8: launch_rows_ch<T, CT, 8>(a, P, block, m); break;
    case 16: launch_rows_ch<T, CT, 16>(a, P, block, m); break;
    default: launch_rows_ch<T, CT, 32>(a, P, block, m); break;
  }
  check_launch(m);
}

// The field's element type T and the type the sweeps compute in: FP64 over
// FP64, FP32 over FP32, or FP64 arithmetic over an FP32 field.
template <typename F>
void with_types(const bfvm_solver* m, F&& f) {
  if (m->precision == BFVM_FP64)
    f(double(), double());
  else if (m->precision == BFVM_FP32_FP64MATH)
    f(float(), double());
  else
    f(float(), float());
}

// The FP64 Thomas tables as the reference holds them, per axis den [n][S],
// cx [n][S], c1 [S] (rebuilt after each Thomas setup): read by the kernels
// that run the reference's own operation sequence.
void ensure_exact_tables(bfvm_solver* m) {
  if (m->cl_tab_ok) return;
  const int ns[3] = {m->nx, m->ny, m->nz};
  for (int a = 0; a < 3; ++a) {
    const size_t nS = (size_t)ns[a] * m->S;
    std::vector<double> t(2 * nS + m->S);
    std::copy(m->h_den[a].begin(), m->h_den[a].end(), t.begin());
    std::copy(m->h_cx[a].begin(), m->h_cx[a].end(), t.begin() + nS);
    std::copy(m->h_c1[a].begin(), m->h_c1[a].end(), t.begin() + 2 * nS);
    upload(m->cl_tab[a], t, m->stream);
  }
  m->cl_tab_ok = true;
}

template <typename T>
void dirichlet_standalone(bfvm_solver* m);
template <typename T>
void bulk_standalone(bfvm_solver* m, double dt);
template <typename T>
void cells_standalone(bfvm_solver* m);

// A sweep of an axis longer than the chunked kernels take: the parts of the
// step fused into the chunked sweeps run as their own kernels around it
// (bulk, cells and the Dirichlet overwrite before, the Dirichlet overwrite
// after), then long_line_kernel over the axis's columns (planes [z0, z1)
// for x and y when z1 >= 0).
template <typename T>
void long_sweep(bfvm_solver* m, int ax, int fuse, int64_t z0, int64_t z1, double dt) {
  ensure_exact_tables(m);
  if (fuse & bfvm::kFuseBulk) bulk_standalone<T>(m, dt);
  if (fuse & bfvm::kFuseCells) cells_standalone<T>(m);
  if ((fuse & bfvm::kFuseDirPro) && m->dir_unique > 0) dirichlet_standalone<T>(m);
  const int64_t S = m->S, nx = m->nx, ny = m->ny, nz = m->nz;
  const int64_t nzp = (m->lod_dims == 2) ? 1 : nz;  // planes swept
  int64_t C, os, ls, ncols, col0 = 0;
  int n;
  if (ax == 0) {
    n = (int)nx, C = S, os = nx * S, ls = S, ncols = ny * nzp * S;
  } else if (ax == 1) {
    n = (int)ny, C = nx * S, os = nx * ny * S, ls = nx * S, ncols = nzp * nx * S;
  } else {
    n = (int)nz, C = nx * ny * S, os = 0, ls = nx * ny * S, ncols = nx * ny * S;
  }
  if (z1 >= 0 && ax < 2) {
    const int64_t per_plane = (ax == 0 ? ny : nx) * S;
    col0 = z0 * per_plane;
    ncols = z1 * per_plane;
  }
  T* p = m->p.as<T>();
  T* out = m->sweep_out ? static_cast<T*>(m->sweep_out) : p;
  const double* t = m->cl_tab[ax].as<double>();
  const int64_t nS = (int64_t)n * S;
  if (ncols > col0) {
    bfvm::long_line_kernel<T><<<(unsigned)blocks_for(ncols - col0, 128), 128, 0, m->stream>>>(
        p, out, col0, ncols, C, os, ls, n, (int)S, t, t + nS, t + 2 * nS);
    check_launch(m);
  }
  if ((fuse & bfvm::kFuseDirEpi) && m->dir_unique > 0) dirichlet_standalone<T>(m);
}

void sweep(bfvm_solver* m, int ax, int fuse, double dt, int64_t z0, int64_t z1) {
  if (long_axis(m, ax)) {
    if (m->precision == BFVM_FP64)
      long_sweep<double>(m, ax, fuse, z0, z1, dt);
    else
      long_sweep<float>(m, ax, fuse, z0, z1, dt);
    return;
  }
  // under AUTO an axis may carry its own kernel choice (bfvm_tune_sweeps)
  const int path =
      (m->path == BFVM_PATH_AUTO && m->axis[ax].kind) ? m->axis[ax].kind : m->path;
  with_types(m, [&](auto t, auto ct) {
    using T = decltype(t);
    using CT = decltype(ct);
    if (path != BFVM_PATH_GENERIC) {
      // build the chunk tables first: the plans size shared memory from them
      chunk_view<CT>(m, ax);
      // AUTO: the register kernel for x (measured fastest there), TMA tiles
      // for y and z
      if (path == BFVM_PATH_AUTO && ax == 0) {
        launch_sweep<T, CT>(m, ax, fuse, dt, z0, z1);
        return;
      }
      const bool want_tma = (path == BFVM_PATH_TMA) || (path == BFVM_PATH_AUTO);
      if (want_tma && ax == 0) {
        const RowsPlan P = plan_rows(m);
        if (P.ok) {
          launch_rows<T, CT>(m, P, fuse, dt, z0, z1);
          return;
        }
        // rows too long for the row kernel: the line kernel, with the
        // Dirichlet overwrites around it (sources fused into the x sweep
        // stay with the kernels that fuse them)
        const LinesPlan L = plan_lines(m, 0);
        if (L.ok && !(fuse & (bfvm::kFuseBulk | bfvm::kFuseCells))) {
          if ((fuse & bfvm::kFuseDirPro) && m->dir_unique > 0) dirichlet_standalone<T>(m);
          launch_lines<T, CT>(m, 0, L, false, z0, z1);
          if ((fuse & bfvm::kFuseDirEpi) && m->dir_unique > 0) dirichlet_standalone<T>(m);
          return;
        }
      } else if (want_tma) {
        const LinesPlan L = plan_lines(m, ax);
        if (L.ok) {
          const bool dir = (ax == 1) && (fuse & bfvm::kFuseDirEpi) && m->seg_dir_y.present;
          launch_lines<T, CT>(m, ax, L, dir, z0, z1);
          return;
        }
      }
      if (launch_direct<T, CT>(m, ax, fuse, dt, z0, z1)) return;
    }
    launch_sweep<T, CT>(m, ax, fuse, dt, z0, z1);
  });
}

void check_status(bfvm_solver* m) {
  int st = 0;
  BFVM_CUDA(cudaMemcpyAsync(&st, m->d_status.ptr, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  BFVM_CUDA(cudaStreamSynchronize(m->stream));
  if (st != 0) {
    BFVM_CUDA(cudaMemsetAsync(m->d_status.ptr, 0, sizeof(int), m->stream));
    throw Error(BFVM_ERR_STATE, "a sweep kernel gave up waiting for its tile copies");
  }
}

void check_lod_mesh(bfvm_solver* m) {
  // BioFVM_solvers.cpp:79-83
  require(m->uniform,
          "Error: This algorithm is written for uniform Cartesian meshes. Try: other solvers!",
          BFVM_ERR_MESH);
}

void bulk_any(bfvm_solver* m, double dt);
void cells_any(bfvm_solver* m);

// One step: bulk -> cells -> LOD_3D (BioFVM_solvers.cpp:175-273), the parts
// selected by flags (diffusion always).  Bulk and cell updates run as their
// own kernels over the sparse lists (they touch only the listed voxels) unless
// fuse_sources folds them into the x sweep's prologue.  The Dirichlet
// overwrites are fused into the sweeps.  ev (optional, 5 events) brackets
// the source kernels, the x, y and z sweeps.
void step_once(bfvm_solver* m, double dt, int flags, cudaEvent_t* ev) {
  check_lod_mesh(m);
  if (!m->setup_done) thomas_setup(m, dt);
  build_all(m);
  if (ev) BFVM_CUDA(cudaEventRecord(ev[0], m->stream));
  int fuse = 0;
  if (m->fuse_sources) {
    if (flags & BFVM_STEP_BULK) fuse |= bfvm::kFuseBulk;
    if (flags & BFVM_STEP_CELLS) fuse |= bfvm::kFuseCells;
  } else {
    if (flags & BFVM_STEP_BULK) bulk_any(m, dt);
    if (flags & BFVM_STEP_CELLS) cells_any(m);
  }
  if (ev) BFVM_CUDA(cudaEventRecord(ev[1], m->stream));
  const int k = m->slab_planes;
  if (k > 0 && k < m->nz && m->lod_dims == 3) {
    // x then y on slabs of k planes: an x line and a y line lie in one z
    // plane, so the y sweep of a slab needs only that slab's x sweep, and a
    // slab small enough for L2 is read back by the y sweep from L2 (the field
    // crosses HBM once for both sweeps instead of twice)
    for (int64_t z0 = 0; z0 < m->nz; z0 += k) {
      const int64_t z1 = std::min<int64_t>(m->nz, z0 + k);
      sweep(m, 0, fuse | bfvm::kFuseDirPro | bfvm::kFuseDirEpi, dt, z0, z1);
      sweep(m, 1, bfvm::kFuseDirEpi, dt, z0, z1);
    }
    // profiles: the x entry holds both sweeps, the y entry nothing
    if (ev) BFVM_CUDA(cudaEventRecord(ev[2], m->stream));
  } else {
    sweep(m, 0, fuse | bfvm::kFuseDirPro | bfvm::kFuseDirEpi, dt);
    if (ev) BFVM_CUDA(cudaEventRecord(ev[2], m->stream));
    sweep(m, 1, bfvm::kFuseDirEpi, dt);
  }
  if (ev) BFVM_CUDA(cudaEventRecord(ev[3], m->stream));
  sweep(m, 2, 0, dt);
  if (ev) BFVM_CUDA(cudaEventRecord(ev[4], m->stream));
}

void diffusion(bfvm_solver* m, double dt) { step_once(m, dt, BFVM_STEP_DIFFUSION, nullptr); }

// diffusion_decay_solver__constant_coefficients_LOD_2D (BioFVM_solvers.cpp:278-427):
// uniform mesh, Dirichlet then x-Thomas, Dirichlet then y-Thomas, on the
// z = 0 plane.
template <typename T>
void dirichlet_standalone(bfvm_solver* m);

void diffusion_2d(bfvm_solver* m, double dt) {
  require(m->uniform,
          "Error: This algorithm is written for uniform Cartesian meshes. Try: something else.",
          BFVM_ERR_MESH);
  struct Restore {
    bfvm_solver* m;
    ~Restore() { m->lod_dims = 3; }
  } restore{m};
  m->lod_dims = 2;
  if (!m->setup_done) thomas_setup(m, dt);
  build_all(m);
  // apply_dirichlet_conditions covers every node, also those off the z = 0
  // plane that the sweeps never touch (:367, :394); the fused overwrites
  // below cover the swept plane.
  if (m->nz > 1 && m->dir_unique > 0) {
    if (m->precision == BFVM_FP64)
      dirichlet_standalone<double>(m);
    else
      dirichlet_standalone<float>(m);
  }
  sweep(m, 0, bfvm::kFuseDirPro | bfvm::kFuseDirEpi, dt);
  sweep(m, 1, 0, dt);
}

template <typename T>
void bulk_standalone(bfvm_solver* m, double dt) {
  const int64_t E = (int64_t)m->bulk_vox.size();
  if (E == 0) return;
  const int64_t work = E * m->S;
  if (m->bulk_rows > 0)
    bfvm::bulk_rows_kernel<T><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
        m->p.as<T>(), m->S, E, m->d_bulk_vox32.as<int>(), m->d_bulk_row.as<int>(),
        m->d_bulk_tab.as<double>(), dt);
  else
    bfvm::bulk_kernel<T><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
        m->p.as<T>(), m->S, E, m->d_bulk_vox.as<int64_t>(), m->d_bulk_st.as<double>(),
        m->d_bulk_su.as<double>(), dt);
  check_launch(m);
}

template <typename T>
void cells_standalone(bfvm_solver* m) {
  const int64_t A = m->n_agents;
  if (A == 0) return;
  const int64_t work = A * m->S;
  bfvm::cells_kernel<T><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
      m->p.as<T>(), m->S, A, m->d_ag_key.as<uint64_t>(), m->d_ag_idx.as<int>(),
      m->d_ag_t1.as<double>(), m->d_ag_t2.as<double>());
  check_launch(m);
}

template <typename T>
void dirichlet_standalone(bfvm_solver* m) {
  if (m->dir_unique == 0) return;
  const int64_t work = m->dir_unique * m->S;
  bfvm::dirichlet_kernel<T><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
      m->p.as<T>(), m->S, m->dir_unique, m->d_dir_vox.as<int64_t>(), m->d_dir_val.as<double>());
  check_launch(m);
}

template <typename T>
void gather(bfvm_solver* m, int64_t count, const int64_t* d_vox, double* d_out) {
  if (count == 0) return;
  const int64_t work = count * m->S;
  bfvm::gather_kernel<T><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
      m->p.as<T>(), m->S, count, d_vox, d_out);
  check_launch(m);
}

void bulk_any(bfvm_solver* m, double dt) {
  if (m->precision == BFVM_FP64)
    bulk_standalone<double>(m, dt);
  else
    bulk_standalone<float>(m, dt);
}

void cells_any(bfvm_solver* m) {
  if (m->precision == BFVM_FP64)
    cells_standalone<double>(m);
  else
    cells_standalone<float>(m);
}

void validate_voxels(const bfvm_solver* m, int64_t count, const int64_t* vox) {
  const int64_t N = m->N();
  for (int64_t e = 0; e < count; ++e)
    if (vox[e] < 0 || vox[e] >= N)  // the message is built only on failure
      throw Error(BFVM_ERR_ARG, "voxel index " + std::to_string(vox[e]) + " outside [0, " +
                                    std::to_string(N) + ")");
}

void resize_common(bfvm_solver* m, int nx, int ny, int nz) {
  require(nx > 0 && ny > 0 && nz > 0, "node counts must be positive");
  require((int64_t)nx * ny * nz * std::max(m->S, 1) < ((int64_t)1 << 40), "mesh too large");
  m->nx = nx;
  m->ny = ny;
  m->nz = nz;
  clear_state_after_resize(m);
}


template void dirichlet_standalone<double>(bfvm_solver* m);

}  // namespace bfvm_rt

using namespace bfvm_rt;

// Upload and download streams of the asynchronous agent exchange and their
// events, created on first use.
void ensure_transfer_streams(bfvm_solver* m) {
  if (m->xf_down_done) return;  // created last
  if (!m->xf_up) BFVM_CUDA(cudaStreamCreateWithFlags(&m->xf_up, cudaStreamNonBlocking));
  if (!m->xf_down) BFVM_CUDA(cudaStreamCreateWithFlags(&m->xf_down, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&m->xf_up_done, &m->xf_spare_free, &m->xf_gathered, &m->xf_down_done})
    if (!*e) BFVM_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
}

// Both transfer streams drained (the host arrays of the asynchronous calls
// are free, their outputs written).
void wait_transfers(bfvm_solver* m) {
  if (m->xf_up_pending) BFVM_CUDA(cudaEventSynchronize(m->xf_up_done));
  if (m->xf_down_pending) BFVM_CUDA(cudaEventSynchronize(m->xf_down_done));
  m->xf_up_pending = m->xf_down_pending = false;
}

// The densities at the agents' voxels into d_gather [A][S] FP64, after any
// copy out of d_gather still running on the download stream.
void gather_agents(bfvm_solver* m) {
  const int64_t A = m->n_agents;
  if (m->xf_down_pending) BFVM_CUDA(cudaStreamWaitEvent(m->stream, m->xf_down_done, 0));
  m->d_gather.ensure(A * m->S * sizeof(double));
  if (m->precision == BFVM_FP64)
    gather<double>(m, A, m->d_ag_vox_orig.as<int64_t>(), m->d_gather.as<double>());
  else
    gather<float>(m, A, m->d_ag_vox_orig.as<int64_t>(), m->d_gather.as<double>());
}

extern "C" {

const char* bfvm_last_error(void) { return g_last_error.c_str(); }
int bfvm_version(void) { return 100; }

int bfvm_create(bfvm_solver** out, int device) {
  return guarded([&] {
    require(out != nullptr, "null output pointer");
    int ndev = 0;
    BFVM_CUDA(cudaGetDeviceCount(&ndev));
    require(device >= 0 && device < ndev, "no CUDA device " + std::to_string(device));
    DeviceGuard dg(device);
    bfvm_solver* m = new bfvm_solver;
    m->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete m;
      throw Error(BFVM_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    }
    m->d_status.ensure(16);
    BFVM_CUDA(cudaMemset(m->d_status.ptr, 0, 16));
    BFVM_CUDA(cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device));
    // Microenvironment(): mesh.resize(1,1,1) (BioFVM_microenvironment.cpp:101)
    // = resize(-0.5, 0.5, ..., 1, 1, 1) (BioFVM_mesh.cpp:924-925), dx = 1.
    resize_common(m, 1, 1, 1);
    *out = m;
  });
}

int bfvm_destroy(bfvm_solver* m) {
  return guarded([&] {
    if (!m) return;
    DeviceGuard dg(m->device);
    cudaStreamSynchronize(m->stream);
    for (cudaStream_t x : {m->xf_up, m->xf_down})
      if (x) cudaStreamSynchronize(x);
    for (DevBuf* d : {&m->xf_vox, &m->xf_t1, &m->xf_t2, &m->xf_key, &m->xf_idx_in, &m->xf_idx,
                      &m->xf_sort_tmp})
      d->release();
    for (cudaEvent_t e : {m->xf_up_done, m->xf_spare_free, m->xf_gathered, m->xf_down_done})
      if (e) cudaEventDestroy(e);
    for (cudaStream_t x : {m->xf_up, m->xf_down})
      if (x) cudaStreamDestroy(x);
    m->p.release();
    for (auto& c : m->coef) c.release();
    m->d_bulk_vox.release();
    m->d_bulk_st.release();
    m->d_bulk_su.release();
    m->d_bulk_vox32.release();
    m->d_bulk_row.release();
    m->d_bulk_tab.release();
    m->seg_bulk.release();
    m->d_dir_vox.release();
    m->d_dir_val.release();
    m->seg_dir_x.release();
    m->seg_dir_y.release();
    m->d_ag_vox_orig.release();
    m->d_ag_t1.release();
    m->d_ag_t2.release();
    m->d_ag_key.release();
    m->d_ag_idx_in.release();
    m->d_ag_idx.release();
    m->d_sort_tmp.release();
    m->d_gather.release();
    m->seg_cells.release();
    m->d_status.release();
    m->d_grad.release();
    adjoint_release(m);
    for (auto& c : m->chunk) c.release();
    for (auto& c : m->chunk_il) c.release();
    for (auto& c : m->chunk_slots) c.release();
    for (auto& c : m->cl_tab) c.release();
    m->d_grid_maps.release();
    cudaStreamDestroy(m->stream);
    delete m;
  });
}

int bfvm_resize_space(bfvm_solver* m, double x0, double x1, double y0, double y1, double z0,
                      double z1, double dx, double dy, double dz) {
  return SOLVER_CALL(m, {
    require(dx > 0 && dy > 0 && dz > 0, "voxel spacing must be positive");
    require(x1 > x0 && y1 > y0 && z1 > z0, "empty domain");
    // BioFVM_mesh.cpp:796-836
    const int nx = bfvm::nodes_from_spacing(x0, x1, dx);
    const int ny = bfvm::nodes_from_spacing(y0, y1, dy);
    const int nz = bfvm::nodes_from_spacing(z0, z1, dz);
    const double tol = 1e-16;
    m->uniform = !(std::fabs(dx - dy) > tol || std::fabs(dy - dz) > tol ||
                   std::fabs(dx - dz) > tol);
    m->dx = dx;
    m->dy = dy;
    m->dz = dz;
    m->dV = dx * dy * dz;
    const double bb[6] = {x0, y0, z0, x1, y1, z1};
    std::copy(bb, bb + 6, m->bbox);
    resize_common(m, nx, ny, nz);
  });
}

int bfvm_resize_space_nodes(bfvm_solver* m, double x0, double x1, double y0, double y1,
                            double z0, double z1, int nx, int ny, int nz) {
  return SOLVER_CALL(m, {
    require(nx > 0 && ny > 0 && nz > 0, "node counts must be positive");
    // BioFVM_mesh.cpp:669-704
    double dx = (x1 - x0) / (double)nx;
    if (nx < 2) dx = 1;
    double dy = (y1 - y0) / (double)ny;
    if (ny < 2) dy = 1;
    double dz = (z1 - z0) / (double)nz;
    if (nz < 2) dz = 1;
    const double tol = 1e-16;
    bool uni = true;
    if (std::fabs(dx - dy) > tol && nx > 1 && ny > 1) uni = false;
    if (std::fabs(dy - dz) > tol && ny > 1 && nz > 1) uni = false;
    if (std::fabs(dx - dz) > tol && nx > 1 && nz > 1) uni = false;
    m->uniform = uni;
    m->dx = dx;
    m->dy = dy;
    m->dz = dz;
    m->dV = dx * dy * dz;
    const double bb[6] = {x0, y0, z0, x1, y1, z1};
    std::copy(bb, bb + 6, m->bbox);
    resize_common(m, nx, ny, nz);
  });
}

int bfvm_set_mesh(bfvm_solver* m, const int* nxyz, const double* geom, int uniform) {
  return SOLVER_CALL(m, {
    require(nxyz != nullptr && geom != nullptr, "null mesh description");
    require(geom[0] > 0 && geom[1] > 0 && geom[2] > 0, "voxel spacing must be positive");
    m->dx = geom[0];
    m->dy = geom[1];
    m->dz = geom[2];
    m->dV = geom[0] * geom[1] * geom[2];
    std::copy(geom + 4, geom + 10, m->bbox);
    m->uniform = uniform != 0;
    resize_common(m, nxyz[0], nxyz[1], nxyz[2]);
  });
}

int bfvm_get_mesh(bfvm_solver* m, int* nxyz, double* geom, int* flags) {
  return SOLVER_CALL(m, {
    if (nxyz) {
      nxyz[0] = m->nx;
      nxyz[1] = m->ny;
      nxyz[2] = m->nz;
    }
    if (geom) {
      geom[0] = m->dx;
      geom[1] = m->dy;
      geom[2] = m->dz;
      geom[3] = m->dV;
      std::copy(m->bbox, m->bbox + 6, geom + 4);
    }
    if (flags) {
      flags[0] = m->uniform ? 1 : 0;
      flags[1] = m->S;
    }
  });
}

int bfvm_resize_densities(bfvm_solver* m, int num_densities) {
  return SOLVER_CALL(m, {
    require(num_densities > 0, "need at least one density");
    m->S = num_densities;
    m->setup_done = false;  // new densities: the next step sets the tables up
    m->D.assign(num_densities, 0.0);
    m->decay.assign(num_densities, 0.0);
    m->d_grad.release();
    m->p.ensure(std::max<size_t>(m->NS() * m->elem(), 16));
    BFVM_CUDA(cudaMemsetAsync(m->p.ptr, 0, m->NS() * m->elem(), m->stream));
    // resize_densities keeps the Dirichlet list but its value vectors no
    // longer match S; the list is cleared so no stale node is applied.
    m->dir_vox.clear();
    m->dir_val.clear();
    m->dir_dirty = true;
    m->bulk_vox.clear();
    m->bulk_st.clear();
    m->bulk_su.clear();
    m->bulk_dirty = true;
    m->n_agents = 0;
    m->ag_dirty = m->ag_seg_dirty = true;
    choose_axes(m);  // the x kernel depends on the number of densities
  });
}

int bfvm_add_density(bfvm_solver* m, double diffusion_coefficient, double decay_rate) {
  return SOLVER_CALL(m, {
    // BioFVM_microenvironment.cpp:404-441: every voxel vector gets one more
    // zero entry; existing densities keep their values.
    const int S0 = m->S, S1 = S0 + 1;
    const int64_t N = m->N();
    DevBuf np;
    np.ensure(std::max<size_t>((size_t)N * S1 * m->elem(), 16));
    BFVM_CUDA(cudaMemsetAsync(np.ptr, 0, (size_t)N * S1 * m->elem(), m->stream));
    BFVM_CUDA(cudaMemcpy2DAsync(np.ptr, S1 * m->elem(), m->p.ptr, S0 * m->elem(),
                                S0 * m->elem(), N, cudaMemcpyDeviceToDevice, m->stream));
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
    m->p.release();
    m->p = np;
    np.ptr = nullptr;
    m->S = S1;
    m->D.push_back(diffusion_coefficient);
    m->decay.push_back(decay_rate);
    // Per-density tables grow with zero entries for the new density.
    auto widen = [&](std::vector<double>& v, double fill) {
      if (v.empty()) return;
      const size_t rows = v.size() / S0;
      std::vector<double> w(rows * S1, fill);
      for (size_t r = 0; r < rows; ++r) std::copy_n(&v[r * S0], S0, &w[r * S1]);
      v.swap(w);
    };
    widen(m->dir_val, 0.0);
    widen(m->bulk_st, 0.0);
    widen(m->bulk_su, 0.0);
    widen_agents(m, S0);
    if (m->d_grad.ptr) {  // gradient vectors keep their values, zeros for the new density
      DevBuf g;
      g.ensure((size_t)N * S1 * 3 * sizeof(double));
      BFVM_CUDA(cudaMemsetAsync(g.ptr, 0, (size_t)N * S1 * 3 * sizeof(double), m->stream));
      BFVM_CUDA(cudaMemcpy2DAsync(g.ptr, S1 * 3 * sizeof(double), m->d_grad.ptr,
                                  S0 * 3 * sizeof(double), S0 * 3 * sizeof(double), N,
                                  cudaMemcpyDeviceToDevice, m->stream));
      BFVM_CUDA(cudaStreamSynchronize(m->stream));
      m->d_grad.release();
      m->d_grad = g;
      g.ptr = nullptr;
    }
    m->dir_dirty = m->bulk_dirty = true;
    m->ag_dirty = m->ag_seg_dirty = true;
    choose_axes(m);  // the x kernel depends on the number of densities
    // The reference keeps its Thomas tables after add_density (sized for the
    // old count; its next solve reads past them).  Here the tables are
    // rebuilt for S1 densities from the setup's own dt and coefficients, so
    // the existing densities keep exactly the coefficients they had and the
    // new one gets its own.
    if (m->setup_done) {
      m->setup_D.push_back(diffusion_coefficient);
      m->setup_decay.push_back(decay_rate);
      std::vector<double> D = m->setup_D, decay = m->setup_decay;
      m->D.swap(D);
      m->decay.swap(decay);
      try {
        thomas_setup(m, m->setup_dt);
      } catch (...) {
        m->D.swap(D);
        m->decay.swap(decay);
        throw;
      }
      m->D.swap(D);
      m->decay.swap(decay);
    }
  });
}

int bfvm_set_density_coefficients(bfvm_solver* m, int index, double diffusion_coefficient,
                                  double decay_rate) {
  return SOLVER_CALL(m, {
    require(index >= 0 && index < m->S, "density index out of range");
    m->D[index] = diffusion_coefficient;
    m->decay[index] = decay_rate;
  });
}

int bfvm_get_num_densities(bfvm_solver* m, int* num_densities) {
  return SOLVER_CALL(m, {
    require(num_densities != nullptr, "null output pointer");
    *num_densities = m->S;
  });
}

int bfvm_set_densities(bfvm_solver* m, const double* host) {
  return SOLVER_CALL(m, {
    require(host != nullptr, "null host buffer");
    const size_t NS = (size_t)m->NS();
    if (m->precision == BFVM_FP64) {
      BFVM_CUDA(cudaMemcpyAsync(m->p.ptr, host, NS * sizeof(double), cudaMemcpyHostToDevice,
                                m->stream));
    } else {
      std::vector<float> tmp(host, host + NS);
      BFVM_CUDA(cudaMemcpyAsync(m->p.ptr, tmp.data(), NS * sizeof(float),
                                cudaMemcpyHostToDevice, m->stream));
    }
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int bfvm_get_densities(bfvm_solver* m, double* host) {
  return SOLVER_CALL(m, {
    require(host != nullptr, "null host buffer");
    check_status(m);
    const size_t NS = (size_t)m->NS();
    if (m->precision == BFVM_FP64) {
      BFVM_CUDA(cudaMemcpyAsync(host, m->p.ptr, NS * sizeof(double), cudaMemcpyDeviceToHost,
                                m->stream));
      BFVM_CUDA(cudaStreamSynchronize(m->stream));
    } else {
      std::vector<float> tmp(NS);
      BFVM_CUDA(cudaMemcpyAsync(tmp.data(), m->p.ptr, NS * sizeof(float),
                                cudaMemcpyDeviceToHost, m->stream));
      BFVM_CUDA(cudaStreamSynchronize(m->stream));
      std::copy(tmp.begin(), tmp.end(), host);
    }
  });
}

int bfvm_get_voxel_densities(bfvm_solver* m, int64_t count, const int64_t* voxels,
                             double* values) {
  return SOLVER_CALL(m, {
    require(count >= 0 && (count == 0 || (voxels && values)), "bad arguments");
    validate_voxels(m, count, voxels);
    if (count == 0) return;
    DevBuf dv, dout;
    dv.ensure(count * sizeof(int64_t));
    dout.ensure(count * m->S * sizeof(double));
    BFVM_CUDA(cudaMemcpyAsync(dv.ptr, voxels, count * sizeof(int64_t), cudaMemcpyHostToDevice,
                              m->stream));
    if (m->precision == BFVM_FP64)
      gather<double>(m, count, dv.as<int64_t>(), dout.as<double>());
    else
      gather<float>(m, count, dv.as<int64_t>(), dout.as<double>());
    BFVM_CUDA(cudaMemcpyAsync(values, dout.ptr, count * m->S * sizeof(double),
                              cudaMemcpyDeviceToHost, m->stream));
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
    dv.release();
    dout.release();
  });
}

int bfvm_set_voxel_densities(bfvm_solver* m, int64_t count, const int64_t* voxels,
                             const double* values) {
  return SOLVER_CALL(m, {
    require(count >= 0 && (count == 0 || (voxels && values)), "bad arguments");
    validate_voxels(m, count, voxels);
    if (count == 0) return;
    DevBuf dv, din;
    dv.ensure(count * sizeof(int64_t));
    din.ensure(count * m->S * sizeof(double));
    BFVM_CUDA(cudaMemcpyAsync(dv.ptr, voxels, count * sizeof(int64_t), cudaMemcpyHostToDevice,
                              m->stream));
    BFVM_CUDA(cudaMemcpyAsync(din.ptr, values, count * m->S * sizeof(double),
                              cudaMemcpyHostToDevice, m->stream));
    const int64_t work = count * m->S;
    if (m->precision == BFVM_FP64)
      bfvm::scatter_kernel<double><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
          m->p.as<double>(), m->S, count, dv.as<int64_t>(), din.as<double>());
    else
      bfvm::scatter_kernel<float><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
          m->p.as<float>(), m->S, count, dv.as<int64_t>(), din.as<double>());
    check_launch(m);
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
    dv.release();
    din.release();
  });
}

int bfvm_device_densities(bfvm_solver* m, void** device_ptr) {
  return SOLVER_CALL(m, {
    require(device_ptr != nullptr, "null output pointer");
    *device_ptr = m->p.ptr;
  });
}

int bfvm_set_bulk_rates(bfvm_solver* m, const double* supply, const double* target,
                        const double* uptake) {
  return SOLVER_CALL(m, {
    const int S = m->S;
    const int64_t N = m->N();
    m->bulk_vox.clear();
    m->bulk_st.clear();
    m->bulk_su.clear();
    std::vector<double> st(S), su(S);
    for (int64_t n = 0; n < N; ++n) {
      const size_t o = (size_t)n * S;
      bfvm::bulk_coefficients(S, supply ? supply + o : nullptr, target ? target + o : nullptr,
                              uptake ? uptake + o : nullptr, st.data(), su.data());
      bool identity = true;
      for (int s = 0; s < S; ++s) identity = identity && st[s] == 0.0 && su[s] == 0.0;
      if (identity) continue;
      m->bulk_vox.push_back(n);
      m->bulk_st.insert(m->bulk_st.end(), st.begin(), st.end());
      m->bulk_su.insert(m->bulk_su.end(), su.begin(), su.end());
    }
    m->bulk_dirty = true;
  });
}

int bfvm_set_bulk_rates_sparse(bfvm_solver* m, int64_t count, const int64_t* voxels,
                               const double* supply, const double* target,
                               const double* uptake) {
  return SOLVER_CALL(m, {
    require(count >= 0 && (count == 0 || voxels), "bad arguments");
    validate_voxels(m, count, voxels);
    const int S = m->S;
    std::vector<int64_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int64_t a, int64_t b) { return voxels[a] < voxels[b]; });
    m->bulk_vox.clear();
    m->bulk_st.clear();
    m->bulk_su.clear();
    std::vector<double> st(S), su(S);
    for (int64_t r = 0; r < count; ++r) {
      const int64_t e = order[r];
      require(r == 0 || voxels[e] != m->bulk_vox.back(), "repeated voxel in bulk list");
      const size_t o = (size_t)e * S;
      bfvm::bulk_coefficients(S, supply ? supply + o : nullptr, target ? target + o : nullptr,
                              uptake ? uptake + o : nullptr, st.data(), su.data());
      m->bulk_vox.push_back(voxels[e]);
      m->bulk_st.insert(m->bulk_st.end(), st.begin(), st.end());
      m->bulk_su.insert(m->bulk_su.end(), su.begin(), su.end());
    }
    m->bulk_dirty = true;
  });
}

int bfvm_add_dirichlet_node(bfvm_solver* m, int64_t voxel, const double* value) {
  return SOLVER_CALL(m, {
    require(value != nullptr, "null value vector");
    validate_voxels(m, 1, &voxel);
    m->dir_vox.push_back(voxel);
    m->dir_val.insert(m->dir_val.end(), value, value + m->S);
    m->dir_dirty = true;
  });
}

int bfvm_update_dirichlet_node(bfvm_solver* m, int64_t voxel, const double* value) {
  return SOLVER_CALL(m, {
    require(value != nullptr, "null value vector");
    validate_voxels(m, 1, &voxel);
    // BioFVM_microenvironment.cpp:153-167: first matching node, else a new one.
    auto it = std::find(m->dir_vox.begin(), m->dir_vox.end(), voxel);
    if (it == m->dir_vox.end()) {
      m->dir_vox.push_back(voxel);
      m->dir_val.insert(m->dir_val.end(), value, value + m->S);
    } else {
      std::copy_n(value, m->S, &m->dir_val[(size_t)(it - m->dir_vox.begin()) * m->S]);
    }
    m->dir_dirty = true;
  });
}

int bfvm_remove_dirichlet_node(bfvm_solver* m, int64_t voxel) {
  return SOLVER_CALL(m, {
    // BioFVM_microenvironment.cpp:169-189 swaps the node with the last one;
    // the reference then pops the value list twice and never the index list
    // (:186-187), which leaves the lists inconsistent.  Here both lists lose
    // exactly the removed node.
    auto it = std::find(m->dir_vox.begin(), m->dir_vox.end(), voxel);
    if (it == m->dir_vox.end()) return;
    const size_t d = (size_t)(it - m->dir_vox.begin()), last = m->dir_vox.size() - 1;
    m->dir_vox[d] = m->dir_vox[last];
    std::copy_n(&m->dir_val[last * m->S], m->S, &m->dir_val[d * m->S]);
    m->dir_vox.pop_back();
    m->dir_val.resize(m->dir_vox.size() * m->S);
    m->dir_dirty = true;
  });
}

int bfvm_clear_dirichlet_nodes(bfvm_solver* m) {
  return SOLVER_CALL(m, {
    m->dir_vox.clear();
    m->dir_val.clear();
    m->dir_dirty = true;
  });
}

int bfvm_get_num_dirichlet_nodes(bfvm_solver* m, int64_t* count) {
  return SOLVER_CALL(m, {
    require(count != nullptr, "null output pointer");
    *count = (int64_t)m->dir_vox.size();
  });
}

int bfvm_set_agents(bfvm_solver* m, int64_t count, const int64_t* voxel, const double* temp1,
                    const double* temp2) {
  return SOLVER_CALL(m, {
    require(count >= 0 && (count == 0 || (voxel && temp1 && temp2)), "bad arguments");
    require(count < ((int64_t)1 << 31), "too many agents");
    validate_voxels(m, count, voxel);
    cudaStream_t st = m->stream;
    const size_t tbytes = (size_t)count * m->S * sizeof(double);
    m->n_agents = 0;
    m->ag_dirty = m->ag_seg_dirty = true;
    if (count > 0) {
      m->d_ag_vox_orig.ensure(count * sizeof(int64_t));
      m->d_ag_t1.ensure(tbytes);
      m->d_ag_t2.ensure(tbytes);
      BFVM_CUDA(cudaMemcpyAsync(m->d_ag_vox_orig.ptr, voxel, count * sizeof(int64_t),
                                cudaMemcpyHostToDevice, st));
      BFVM_CUDA(cudaMemcpyAsync(m->d_ag_t1.ptr, temp1, tbytes, cudaMemcpyHostToDevice, st));
      BFVM_CUDA(cudaMemcpyAsync(m->d_ag_t2.ptr, temp2, tbytes, cudaMemcpyHostToDevice, st));
      // the caller may reuse its arrays once this call returns
      BFVM_CUDA(cudaStreamSynchronize(st));
    }
    m->n_agents = count;
  });
}

int bfvm_get_agent_densities(bfvm_solver* m, double* values) {
  return SOLVER_CALL(m, {
    const int64_t A = m->n_agents;
    if (A == 0) return;
    require(values != nullptr, "null output buffer");
    gather_agents(m);
    BFVM_CUDA(cudaMemcpyAsync(values, m->d_gather.ptr, A * m->S * sizeof(double),
                              cudaMemcpyDeviceToHost, m->stream));
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int bfvm_set_agents_async(bfvm_solver* m, int64_t count, const int64_t* voxel,
                          const double* temp1, const double* temp2) {
  return SOLVER_CALL(m, {
    require(count >= 0 && (count == 0 || (voxel && temp1 && temp2)), "bad arguments");
    require(count < ((int64_t)1 << 31), "too many agents");
    validate_voxels(m, count, voxel);
    ensure_transfer_streams(m);
    cudaStream_t up = m->xf_up;
    // the spare set is still read by the steps enqueued before it was swapped out
    if (m->xf_spare_recorded) BFVM_CUDA(cudaStreamWaitEvent(up, m->xf_spare_free, 0));
    if (count > 0) {
      const size_t tbytes = (size_t)count * m->S * sizeof(double);
      m->xf_vox.ensure(count * sizeof(int64_t));
      m->xf_t1.ensure(tbytes);
      m->xf_t2.ensure(tbytes);
      BFVM_CUDA(cudaMemcpyAsync(m->xf_vox.ptr, voxel, count * sizeof(int64_t),
                                cudaMemcpyHostToDevice, up));
      BFVM_CUDA(cudaMemcpyAsync(m->xf_t1.ptr, temp1, tbytes, cudaMemcpyHostToDevice, up));
      BFVM_CUDA(cudaMemcpyAsync(m->xf_t2.ptr, temp2, tbytes, cudaMemcpyHostToDevice, up));
      sort_agents(count, m->N(), m->xf_vox.as<uint64_t>(), m->xf_key, m->xf_idx_in, m->xf_idx,
                  m->xf_sort_tmp, up, m);
    }
    BFVM_CUDA(cudaEventRecord(m->xf_up_done, up));
    m->xf_up_pending = true;
    // the current set becomes the spare once the work enqueued so far is done;
    // work enqueued from here on reads the new set after its upload
    BFVM_CUDA(cudaEventRecord(m->xf_spare_free, m->stream));
    m->xf_spare_recorded = true;
    BFVM_CUDA(cudaStreamWaitEvent(m->stream, m->xf_up_done, 0));
    std::swap(m->d_ag_vox_orig, m->xf_vox);
    std::swap(m->d_ag_t1, m->xf_t1);
    std::swap(m->d_ag_t2, m->xf_t2);
    std::swap(m->d_ag_key, m->xf_key);
    std::swap(m->d_ag_idx_in, m->xf_idx_in);
    std::swap(m->d_ag_idx, m->xf_idx);
    std::swap(m->d_sort_tmp, m->xf_sort_tmp);
    m->n_agents = count;
    m->ag_dirty = false;  // sorted on the upload stream
    m->ag_seg_dirty = true;
    ++m->lists_version;
  });
}

int bfvm_get_agent_densities_async(bfvm_solver* m, double* values) {
  return SOLVER_CALL(m, {
    const int64_t A = m->n_agents;
    if (A == 0) return;
    require(values != nullptr, "null output buffer");
    ensure_transfer_streams(m);
    gather_agents(m);
    BFVM_CUDA(cudaEventRecord(m->xf_gathered, m->stream));
    BFVM_CUDA(cudaStreamWaitEvent(m->xf_down, m->xf_gathered, 0));
    BFVM_CUDA(cudaMemcpyAsync(values, m->d_gather.ptr, A * m->S * sizeof(double),
                              cudaMemcpyDeviceToHost, m->xf_down));
    BFVM_CUDA(cudaEventRecord(m->xf_down_done, m->xf_down));
    m->xf_down_pending = true;
  });
}

int bfvm_wait_transfers(bfvm_solver* m) {
  return SOLVER_CALL(m, { wait_transfers(m); });
}

int bfvm_simulate_bulk_sources_and_sinks(bfvm_solver* m, double dt) {
  return SOLVER_CALL(m, {
    build_bulk(m);
    bulk_any(m, dt);
  });
}

int bfvm_simulate_cell_sources_and_sinks(bfvm_solver* m, double dt) {
  (void)dt;  // unused by the reference as well (BioFVM_basic_agent.cpp:229)
  return SOLVER_CALL(m, {
    build_agents(m);
    cells_any(m);
  });
}

int bfvm_simulate_diffusion_decay(bfvm_solver* m, double dt) {
  return SOLVER_CALL(m, diffusion(m, dt));
}

int bfvm_simulate_diffusion_decay_2d(bfvm_solver* m, double dt) {
  return SOLVER_CALL(m, diffusion_2d(m, dt));
}

int bfvm_apply_dirichlet_conditions(bfvm_solver* m) {
  return SOLVER_CALL(m, {
    build_dirichlet(m);
    if (m->precision == BFVM_FP64)
      dirichlet_standalone<double>(m);
    else
      dirichlet_standalone<float>(m);
  });
}

namespace bfvm_rt {

constexpr int kClusterMaxN = 64;                  // points per axis (registers per line)
constexpr size_t kClusterSlabBytes = 200 * 1024;  // field in shared memory per block
constexpr size_t kClusterSmemMax = 224 * 1024;    // with the staged Dirichlet nodes

// Blocks of the cluster that holds the whole field (1, 2, 4 or 8), or 0 when
// bfvm_step cannot run this solver's steps in one cluster.
int cluster_blocks(const bfvm_solver* m) {
  if (!m->cluster_steps || m->path != BFVM_PATH_AUTO || m->precision != BFVM_FP64 ||
      m->lod_dims != 3 || !m->uniform || m->fuse_sources || m->slab_planes > 0)
    return 0;
  if (m->nx > kClusterMaxN || m->ny > kClusterMaxN || m->nz > kClusterMaxN) return 0;
  for (int cl : {1, 2, 4, 8}) {
    const int64_t pz = (m->nz + cl - 1) / cl;
    if ((size_t)(pz * m->nx * m->ny * m->S) * sizeof(double) <= kClusterSlabBytes) return cl;
  }
  return 0;
}

// nsteps whole steps (bulk -> cells -> LOD_3D) in one cluster launch.
void cluster_run(bfvm_solver* m, double dt, int nsteps, int flags, int cl) {
  ensure_exact_tables(m);
  bfvm::ClusterStepArgs a{};
  a.p = m->p.as<double>();
  a.nx = m->nx;
  a.ny = m->ny;
  a.nz = m->nz;
  a.S = m->S;
  a.pz = (m->nz + cl - 1) / cl;
  a.nsteps = nsteps;
  a.dt = dt;
  a.bulk = (flags & BFVM_STEP_BULK) && !m->bulk_vox.empty();
  a.cells = (flags & BFVM_STEP_CELLS) && m->n_agents > 0;
  a.diffusion = true;
  const int ns[3] = {m->nx, m->ny, m->nz};
  for (int ax = 0; ax < 3; ++ax) {
    const double* t = m->cl_tab[ax].as<double>();
    const size_t nS = (size_t)ns[ax] * m->S;
    a.den[ax] = t;
    a.cx[ax] = t + nS;
    a.c1[ax] = t + 2 * nS;
  }
  a.nbulk = (int64_t)m->bulk_vox.size();
  a.bulk_vox = m->d_bulk_vox.as<int64_t>();
  a.bulk_st = m->d_bulk_st.as<double>();
  a.bulk_su = m->d_bulk_su.as<double>();
  a.nagents = m->n_agents;
  a.ag_key = m->d_ag_key.as<uint64_t>();
  a.ag_idx = m->d_ag_idx.as<int>();
  a.ag_t1 = m->d_ag_t1.as<double>();
  a.ag_t2 = m->d_ag_t2.as<double>();
  a.ndir = m->dir_unique;
  a.dir_vox = m->d_dir_vox.as<int64_t>();
  a.dir_val = m->d_dir_val.as<double>();
  // each block's Dirichlet nodes and bulk entries (both lists ascending in
  // voxel) are contiguous: [lo, hi) per block; the Dirichlet nodes are staged
  // in the block's shared memory for the whole launch when they fit
  const int64_t plane = (int64_t)m->nx * m->ny;
  int dir_max = 0;
  for (int r = 0; r < cl; ++r) {
    const int64_t v0 = std::min<int64_t>(m->nz, (int64_t)r * a.pz) * plane;
    const int64_t v1 = std::min<int64_t>(m->nz, (int64_t)(r + 1) * a.pz) * plane;
    const auto& dv = m->dir_sorted;
    a.dir_lo[r] = (int)(std::lower_bound(dv.begin(), dv.end(), v0) - dv.begin());
    a.dir_hi[r] = (int)(std::lower_bound(dv.begin(), dv.end(), v1) - dv.begin());
    dir_max = std::max(dir_max, a.dir_hi[r] - a.dir_lo[r]);
    const auto& bv = m->bulk_vox;
    a.bulk_lo[r] = std::lower_bound(bv.begin(), bv.end(), v0) - bv.begin();
    a.bulk_hi[r] = std::lower_bound(bv.begin(), bv.end(), v1) - bv.begin();
  }
  const size_t slab_bytes = (size_t)a.pz * m->nx * m->ny * m->S * sizeof(double);
  const size_t dir_bytes = (size_t)dir_max * (m->S * sizeof(double) + sizeof(int));
  a.dir_staged = slab_bytes + dir_bytes <= kClusterSmemMax;
  const size_t smem = slab_bytes + (a.dir_staged ? dir_bytes : 0) + 16;
  auto k = bfvm::cluster_steps_kernel<kClusterMaxN>;
  allow_smem((const void*)k, m->device, smem);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cl);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = m->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BFVM_CUDA(cudaLaunchKernelEx(&cfg, k, a));
  check_launch(m);
}

constexpr int kGridMaxN = 64;              // points per axis (registers per line)
// voxel-densities: measured faster than the sweep kernels up to 2^19 (18.7 vs
// 26.7 us/step at 50^3 x 1, 24.8 vs 27.2 at 50^3 x 4), even at 2^20
constexpr int64_t kGridMaxVS = 1 << 19;
constexpr int kGridThreads = 128;
constexpr size_t kGridSmem = (size_t)4 * kGridThreads * sizeof(double);  // chunk carries

// Tiles of the widest phase of grid steps with ch-point chunks (TW = threads
// / chunks columns per tile).
int64_t grid_tiles(const bfvm_solver* m, int ch) {
  const int64_t N = (int64_t)m->nx * m->ny * m->nz;
  const int ns[3] = {m->nx, m->ny, m->nz};
  int64_t tiles = 1;
  for (int ax = 0; ax < 3; ++ax) {
    const int nc = (ns[ax] + ch - 1) / ch;
    const int64_t tw = kGridThreads / nc;
    tiles = std::max(tiles, (N / ns[ax] * m->S + tw - 1) / tw);
  }
  return tiles;
}

// Blocks of the cooperative launch that runs this solver's steps in one
// launch, or 0 when bfvm_step uses the sweep kernels (or the cluster).  *ch:
// the chunk length, 4 when the widest phase fits one wave of resident blocks
// (shorter chains, measured faster: 50^3 x 1 19.9 -> 17.8 us/step, 32^3 x 8
// 21.5 -> 16.8), else 8 (50^3 x 4: 27.3 us/step, 33.4 with 4-point chunks in
// two waves).
int grid_blocks(bfvm_solver* m, int* ch = nullptr) {
  if (!m->grid_steps || m->path != BFVM_PATH_AUTO || m->precision != BFVM_FP64 ||
      m->lod_dims != 3 || !m->uniform || m->fuse_sources || m->slab_planes > 0)
    return 0;
  if (m->nx > kGridMaxN || m->ny > kGridMaxN || m->nz > kGridMaxN) return 0;
  if ((int64_t)m->NS() > kGridMaxVS || cluster_blocks(m) > 0) return 0;
  if (m->grid_per_sm[0] == 0) {
    int coop = 0;
    BFVM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, m->device));
    int per4 = 0, per8 = 0;
    if (coop) {
      allow_smem((const void*)bfvm::grid_steps_kernel<4>, m->device, kGridSmem);
      allow_smem((const void*)bfvm::grid_steps_kernel<8>, m->device, kGridSmem);
      BFVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per4, bfvm::grid_steps_kernel<4>, kGridThreads, kGridSmem));
      BFVM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per8, bfvm::grid_steps_kernel<8>, kGridThreads, kGridSmem));
    }
    m->grid_per_sm[0] = per4 > 0 ? per4 : -1;
    m->grid_per_sm[1] = per8 > 0 ? per8 : -1;
  }
  const int64_t sources =
      (((int64_t)m->bulk_vox.size() + m->n_agents) * m->S + kGridThreads - 1) / kGridThreads;
  for (int i = 0; i < 2; ++i) {
    const int c = i == 0 ? 4 : 8;
    if (m->grid_per_sm[i] < 0) continue;
    const int64_t wave = (int64_t)m->grid_per_sm[i] * m->num_sms;
    const int64_t tiles = grid_tiles(m, c);
    if (tiles <= wave || c == 8) {
      if (ch) *ch = c;
      return (int)std::min<int64_t>(std::max(tiles, sources), wave);
    }
  }
  return 0;
}

// nsteps whole steps (bulk -> cells -> LOD_3D) in one cooperative launch.
void grid_run(bfvm_solver* m, double dt, int nsteps, int flags, int blocks, int ch) {
  const int S = m->S;
  // scratch: Dirichlet values [N][S] (doubles first), line masks of the x, y
  // and z lines, bulk and agent maps [N] each
  const int64_t N = m->N();
  const int64_t lx = N / m->nx, ly = N / m->ny, lz = N / m->nz;
  const size_t field_b = (size_t)N * S * sizeof(double);
  const size_t masks_b = (size_t)(lx + ly + lz) * sizeof(uint64_t);
  const void* before = m->d_grid_maps.ptr;
  m->d_grid_maps.ensure(field_b + masks_b + (size_t)2 * N * sizeof(int));
  unsigned char* base = m->d_grid_maps.as<unsigned char>();
  double* dir_field = reinterpret_cast<double*>(base);
  unsigned long long* mx = reinterpret_cast<unsigned long long*>(base + field_b);
  unsigned long long* my = mx + lx;
  unsigned long long* mz = my + ly;
  int* maps = reinterpret_cast<int*>(base + field_b + masks_b);
  const int64_t nbulk = (int64_t)m->bulk_vox.size();
  // the maps are rebuilt only when a list changed since they were built (or
  // the buffer moved, or the number of densities changed)
  const bool rebuild = m->grid_maps_version != m->lists_version || before != m->d_grid_maps.ptr ||
                       m->grid_maps_S != S;
  if (rebuild) {
    BFVM_CUDA(cudaMemsetAsync(mx, 0, masks_b, m->stream));
    BFVM_CUDA(cudaMemsetAsync(maps, 0xFF, (size_t)2 * N * sizeof(int), m->stream));
    m->grid_maps_version = m->lists_version;
    m->grid_maps_S = S;
  }
  const int64_t most = std::max({nbulk, m->n_agents, m->dir_unique});
  if (rebuild && most > 0) {
    bfvm::grid_maps_kernel<<<(unsigned)blocks_for(most, 256), 256, 0, m->stream>>>(
        maps, maps + N, nbulk, m->d_bulk_vox.as<int64_t>(), m->n_agents,
        m->d_ag_key.as<uint64_t>(), m->dir_unique, m->d_dir_vox.as<int64_t>(),
        m->d_dir_val.as<double>(), mx, my, mz, dir_field, m->nx, m->ny, S);
    check_launch(m);
  }
  bfvm::GridStepArgs a{};
  a.p = m->p.as<double>();
  a.nx = m->nx;
  a.ny = m->ny;
  a.nz = m->nz;
  a.S = S;
  a.nsteps = nsteps;
  a.dt = dt;
  a.bulk = (flags & BFVM_STEP_BULK) && nbulk > 0;
  a.cells = (flags & BFVM_STEP_CELLS) && m->n_agents > 0;
  for (int ax = 0; ax < 3; ++ax) a.coef[ax] = coef_view<double>(m, ax);
  a.bulk_map = maps;
  a.ag_map = maps + N;
  a.dirichlet = m->dir_unique > 0;
  a.dir_mask[0] = mx;
  a.dir_mask[1] = my;
  a.dir_mask[2] = mz;
  a.dir_field = dir_field;
  a.nbulk = nbulk;
  a.bulk_vox = m->d_bulk_vox.as<int64_t>();
  a.bulk_st = m->d_bulk_st.as<double>();
  a.bulk_su = m->d_bulk_su.as<double>();
  a.nagents = m->n_agents;
  a.ag_key = m->d_ag_key.as<uint64_t>();
  a.ag_idx = m->d_ag_idx.as<int>();
  a.ag_t1 = m->d_ag_t1.as<double>();
  a.ag_t2 = m->d_ag_t2.as<double>();
  void* params[] = {&a};
  const void* k = ch == 4 ? (const void*)bfvm::grid_steps_kernel<4>
                          : (const void*)bfvm::grid_steps_kernel<8>;
  BFVM_CUDA(cudaLaunchCooperativeKernel(k, dim3((unsigned)blocks), dim3(kGridThreads), params,
                                        kGridSmem, m->stream));
  check_launch(m);
}

}  // namespace bfvm_rt

int bfvm_set_grid_steps(bfvm_solver* m, int enable) {
  return SOLVER_CALL(m, { m->grid_steps = enable ? 1 : 0; });
}

int bfvm_get_grid_steps(bfvm_solver* m, int* blocks) {
  return SOLVER_CALL(m, {
    require(blocks != nullptr, "null output pointer");
    *blocks = grid_blocks(m);
  });
}

int bfvm_set_cluster_steps(bfvm_solver* m, int enable) {
  return SOLVER_CALL(m, { m->cluster_steps = enable ? 1 : 0; });
}

int bfvm_get_cluster_steps(bfvm_solver* m, int* blocks) {
  return SOLVER_CALL(m, {
    require(blocks != nullptr, "null output pointer");
    *blocks = cluster_blocks(m);
  });
}

int bfvm_step(bfvm_solver* m, double dt, int nsteps, int flags) {
  return SOLVER_CALL(m, {
    require(nsteps >= 0, "negative step count");
    require(m->zs_ranks == 0 || nsteps <= 1 || !(flags & BFVM_STEP_DIFFUSION),
            "a z slab takes one diffusion step per call (bfvm_zslab_fixup joins the slabs "
            "after each)");
    require((flags & ~BFVM_STEP_ALL) == 0, "unknown step flags");
    if (!(flags & BFVM_STEP_DIFFUSION)) {
      // No sweep to fuse into: the per-voxel kernels alone.
      build_bulk(m);
      build_agents(m);
      for (int it = 0; it < nsteps; ++it) {
        if (flags & BFVM_STEP_BULK) bulk_any(m, dt);
        if (flags & BFVM_STEP_CELLS) cells_any(m);
      }
      return;
    }
    const int cl = cluster_blocks(m);
    if (cl > 0 && nsteps > 0) {
      check_lod_mesh(m);
      if (!m->setup_done) thomas_setup(m, dt);
      build_all(m);
      cluster_run(m, dt, nsteps, flags, cl);
      return;
    }
    int gch = 8;
    const int gb = nsteps > 0 ? grid_blocks(m, &gch) : 0;
    if (gb > 0) {
      check_lod_mesh(m);
      if (!m->setup_done) thomas_setup(m, dt);
      build_all(m);
      grid_run(m, dt, nsteps, flags, gb, gch);
      return;
    }
    for (int it = 0; it < nsteps; ++it) step_once(m, dt, flags, nullptr);
  });
}

void ensure_gradients(bfvm_solver* m) {
  const size_t bytes = (size_t)m->NS() * 3 * sizeof(double);
  if (m->d_grad.ptr && m->d_grad.bytes >= bytes) return;
  m->d_grad.ensure(std::max<size_t>(bytes, 16));
  BFVM_CUDA(cudaMemsetAsync(m->d_grad.ptr, 0, bytes, m->stream));
}

int bfvm_compute_all_gradient_vectors(bfvm_solver* m) {
  return SOLVER_CALL(m, {
    ensure_gradients(m);
    // the reference divides by 2*dx, 2*dy, 2*dz (:704-713)
    const double two_dx = m->dx * 2.0, two_dy = m->dy * 2.0, two_dz = m->dz * 2.0;
    const int64_t work = m->NS();
    const bool rows = m->ny <= 65535 && m->nz <= 65535 && (int64_t)m->nx * m->S < (1 << 30);
    const dim3 rgrid((unsigned)blocks_for((int64_t)m->nx * m->S, 256), m->ny, m->nz);
    with_types(m, [&](auto t, auto) {
      using T = decltype(t);
      if (rows)
        bfvm::gradient_rows_kernel<T><<<rgrid, 256, 0, m->stream>>>(
            m->p.as<T>(), m->nx, m->ny, m->nz, m->S, two_dx, two_dy, two_dz,
            m->d_grad.as<double>());
      else
        bfvm::gradient_kernel<T><<<(unsigned)blocks_for(work, 256), 256, 0, m->stream>>>(
            m->p.as<T>(), m->nx, m->ny, m->nz, m->S, two_dx, two_dy, two_dz,
            m->d_grad.as<double>());
    });
    check_launch(m);
  });
}

int bfvm_get_gradient_vectors(bfvm_solver* m, double* out) {
  return SOLVER_CALL(m, {
    require(out != nullptr, "null output buffer");
    ensure_gradients(m);
    BFVM_CUDA(cudaMemcpyAsync(out, m->d_grad.ptr, (size_t)m->NS() * 3 * sizeof(double),
                              cudaMemcpyDeviceToHost, m->stream));
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
  });
}

int bfvm_device_gradients(bfvm_solver* m, void** ptr) {
  return SOLVER_CALL(m, {
    require(ptr != nullptr, "null output pointer");
    ensure_gradients(m);
    *ptr = m->d_grad.ptr;
  });
}

int bfvm_set_z_slab(bfvm_solver* m, int nranks, const int* bounds, int rank) {
  return SOLVER_CALL(m, {
    require(nranks >= 0 && nranks <= kZSlabMaxRanks,
            "nranks must be in [0, " + std::to_string(kZSlabMaxRanks) + "]");
    if (nranks == 0) {
      m->zs_ranks = 0;
      m->zs_bounds.clear();
      m->setup_done = false;
      return;
    }
    require(bounds != nullptr && rank >= 0 && rank < nranks, "bad arguments");
    require(bounds[0] == 0, "the first slab starts at plane 0");
    for (int r = 0; r < nranks; ++r)
      require(bounds[r + 1] > bounds[r], "every slab holds at least one plane");
    require(bounds[rank + 1] - bounds[rank] == m->nz,
            "this solver's mesh must have its slab's " +
                std::to_string(bounds[rank + 1] - bounds[rank]) + " planes (it has " +
                std::to_string(m->nz) + ")");
    m->zs_ranks = nranks;
    m->zs_rank = rank;
    m->zs_bounds.assign(bounds, bounds + nranks + 1);
    m->setup_done = false;  // the z coefficients are the whole line's rows
  });
}

int bfvm_zslab_fixup(bfvm_solver* m, const double* planes) {
  return SOLVER_CALL(m, {
    require(m->zs_ranks > 0, "not a z slab (bfvm_set_z_slab)", BFVM_ERR_STATE);
    require(m->setup_done, "no step ran yet", BFVM_ERR_STATE);
    require(m->precision == BFVM_FP64, "z slabs are FP64", BFVM_ERR_STATE);
    require(planes != nullptr, "null planes");
    const int64_t C = (int64_t)m->nx * m->ny * m->S;
    const unsigned grid = (unsigned)blocks_for(C, 128);
    const double* cst = m->zs_const.as<double>();
    const double* pt = m->zs_pt.as<double>();
    if (m->zs_ranks <= 8)
      bfvm::zslab_fixup_kernel<8><<<grid, 128, 0, m->stream>>>(
          m->p.as<double>(), C, m->S, m->nz, m->zs_ranks, m->zs_rank, planes, cst, pt);
    else
      bfvm::zslab_fixup_kernel<kZSlabMaxRanks><<<grid, 128, 0, m->stream>>>(
          m->p.as<double>(), C, m->S, m->nz, m->zs_ranks, m->zs_rank, planes, cst, pt);
    check_launch(m);
  });
}

int bfvm_reset_diffusion_setup(bfvm_solver* m) {
  return SOLVER_CALL(m, { m->setup_done = false; });
}

int bfvm_set_precision(bfvm_solver* m, int precision) {
  return SOLVER_CALL(m, {
    require(precision == BFVM_FP64 || precision == BFVM_FP32 || precision == BFVM_FP32_FP64MATH,
            "precision must be BFVM_FP64, BFVM_FP32 or BFVM_FP32_FP64MATH");
    if (precision == m->precision) return;
    const bool was64 = m->precision == BFVM_FP64, is64 = precision == BFVM_FP64;
    if (was64 != is64) {  // the field changes element type
      const int64_t NS = m->NS();
      DevBuf np;
      np.ensure(std::max<size_t>(NS * (is64 ? 8 : 4), 16));
      if (NS > 0) {
        if (!is64)
          bfvm::convert_kernel<float, double>
              <<<(unsigned)blocks_for(NS, 256), 256, 0, m->stream>>>(np.as<float>(),
                                                                   m->p.as<double>(), NS);
        else
          bfvm::convert_kernel<double, float>
              <<<(unsigned)blocks_for(NS, 256), 256, 0, m->stream>>>(np.as<double>(),
                                                                   m->p.as<float>(), NS);
        check_launch(m);
      }
      BFVM_CUDA(cudaStreamSynchronize(m->stream));
      m->p.release();
      m->p = np;
      np.ptr = nullptr;
    }
    m->precision = precision;
    m->setup_done = false;  // coefficient tables are kept in the sweeps' arithmetic type
    choose_axes(m);
    // segment lists depend on the chunk lengths
    m->bulk_dirty = m->dir_dirty = m->ag_seg_dirty = true;
  });
}

int bfvm_selftest_bounded_wait(int device, int64_t limit_ns, int* gave_up, double* waited_ms) {
  return guarded([&] {
    require(gave_up != nullptr && waited_ms != nullptr, "null output pointer");
    require(limit_ns >= 1000 && limit_ns <= (int64_t)bfvm::tma::kWaitLimitNs,
            "limit_ns must be in [1e3, 2e9]");
    int ndev = 0;
    BFVM_CUDA(cudaGetDeviceCount(&ndev));
    require(device >= 0 && device < ndev, "no CUDA device " + std::to_string(device));
    DeviceGuard dg(device);
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DevBuf status;
    struct Release {
      cudaStream_t& st;
      cudaEvent_t& e0;
      cudaEvent_t& e1;
      ~Release() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (st) cudaStreamDestroy(st);
      }
    } release{st, e0, e1};
    BFVM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    BFVM_CUDA(cudaEventCreate(&e0));
    BFVM_CUDA(cudaEventCreate(&e1));
    status.ensure(sizeof(int));
    BFVM_CUDA(cudaMemsetAsync(status.ptr, 0, sizeof(int), st));
    BFVM_CUDA(cudaEventRecord(e0, st));
    bfvm::bounded_wait_selftest_kernel<<<1, 32, 0, st>>>((unsigned long long)limit_ns,
                                                        status.as<int>());
    BFVM_CUDA(cudaGetLastError());
    BFVM_CUDA(cudaEventRecord(e1, st));
    int h = 0;
    BFVM_CUDA(cudaMemcpyAsync(&h, status.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    BFVM_CUDA(cudaStreamSynchronize(st));
    float ms = 0;
    BFVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *gave_up = h;
    *waited_ms = ms;
  });
}

int bfvm_set_slab_planes(bfvm_solver* m, int planes) {
  return SOLVER_CALL(m, {
    require(planes >= 0, "planes must be >= 0");
    m->slab_planes = planes;
  });
}

int bfvm_get_slab_planes(bfvm_solver* m, int* planes) {
  return SOLVER_CALL(m, {
    require(planes != nullptr, "null output pointer");
    *planes = m->slab_planes;
  });
}

int bfvm_set_sweep_config(bfvm_solver* m, int axis, int chunk, int columns, int min_blocks) {
  return SOLVER_CALL(m, {
    require(axis >= 0 && axis < 3, "axis must be 0, 1 or 2");
    require(chunk == 8 || chunk == 16 || chunk == 32, "chunk must be 8, 16 or 32");
    require(columns == 8 || columns == 16 || columns == 32 || columns == 64,
            "columns must be 8, 16, 32 or 64");
    require(min_blocks == 1 || min_blocks == 2, "min_blocks must be 1 or 2");
    const int ns[3] = {m->nx, m->ny, m->nz};
    const int nc = (ns[axis] + chunk - 1) / chunk;
    require(nc * columns <= bfvm::sweep_max_threads(chunk),
            "chunks x columns exceeds the block size of the sweep kernel (512 threads, 256 "
            "with 32-point chunks)");
    Axis& A = m->axis[axis];
    if (A.ch != chunk) m->bulk_dirty = m->dir_dirty = m->ag_seg_dirty = true;
    A.ch = chunk;
    A.tw = columns;
    A.minb = min_blocks;
    A.kind = 0;
    A.stages = 0;
    A.user = true;
  });
}

}  // extern "C"

namespace bfvm_rt {

// Times every kernel choice of each axis on this solver's own data and keeps
// the fastest (the field is saved before and restored after).
void tune_sweeps(bfvm_solver* m, double dt, int reps) {
  require(reps >= 1 && reps <= 100, "reps must be in [1, 100]");
  check_lod_mesh(m);
  if (!m->setup_done) thomas_setup(m, dt);
  build_all(m);
  const size_t bytes = m->NS() * m->elem();
  DevBuf save;
  save.ensure(std::max<size_t>(bytes, 16));
  BFVM_CUDA(cudaMemcpyAsync(save.ptr, m->p.ptr, bytes, cudaMemcpyDeviceToDevice, m->stream));
  const int saved_path = m->path;
  const int saved_slab = m->slab_planes;
  const int saved_fuse = m->fuse_sources;
  m->path = BFVM_PATH_AUTO;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  BFVM_CUDA(cudaEventCreate(&e0));
  BFVM_CUDA(cudaEventCreate(&e1));
  struct Choice {
    int kind, ch, tw, stages, minb, build;
  };
  const int ns[3] = {m->nx, m->ny, m->nz};
  const int fuses[3] = {bfvm::kFuseDirPro | bfvm::kFuseDirEpi, bfvm::kFuseDirEpi, 0};
  try {
    for (int ax = 0; ax < 3; ++ax) {
      if (long_axis(m, ax)) continue;  // one kernel runs it
      std::vector<Choice> cand;
      for (int ch : {8, 16, 32}) {
        const int nc = (ns[ax] + ch - 1) / ch;
        if (nc > 64) continue;
        for (int tw : {32, 16, 8})
          if (nc * tw <= bfvm::sweep_max_threads(ch))
            cand.push_back({BFVM_PATH_GENERIC, ch, tw, 0, 1, 0});
        // the line kernel also takes 17-32 chunks of 32 points (x: where the
        // rows are too long for the row kernel)
        if (nc <= 16 || (ch == 32 && nc <= 32))
          cand.push_back({BFVM_PATH_TMA, ch, 16, 0, 1, 0});
        // the row kernel (x) with a ring of three tiles, and at 32-point
        // chunks compiled for two blocks per SM or for this density count
        // (interleaved or planar tables; the plan falls back to the general
        // build where these do not apply)
        if (ax == 0 && nc <= 16) cand.push_back({BFVM_PATH_TMA, ch, 16, 3, 1, 0});
        if (ax == 0 && nc <= 16 && ch == 32) {
          cand.push_back({BFVM_PATH_TMA, ch, 16, 0, 2, 0});
          if (row_build_count(m->S)) {
            cand.push_back({BFVM_PATH_TMA, ch, 16, 0, 1, 1});
            cand.push_back({BFVM_PATH_TMA, ch, 16, 0, 1, 2});
          }
        }
        if (nc <= 16) cand.push_back({BFVM_PATH_DIRECT, ch, 16, 0, 1, 0});
      }
      Axis best = m->axis[ax];
      float best_ms = 1e30f;
      for (const Choice& c : cand) {
        Axis& A = m->axis[ax];
        if (A.ch != c.ch) m->bulk_dirty = m->dir_dirty = m->ag_seg_dirty = true;
        A.ch = c.ch;
        A.tw = c.tw;
        A.minb = c.minb;
        A.kind = c.kind;
        A.stages = c.stages;
        A.build = c.build;
        A.user = true;
        build_all(m);
        sweep(m, ax, fuses[ax], dt);  // warm-up: tables and plans
        BFVM_CUDA(cudaEventRecord(e0, m->stream));
        for (int r = 0; r < reps; ++r) sweep(m, ax, fuses[ax], dt);
        BFVM_CUDA(cudaEventRecord(e1, m->stream));
        BFVM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BFVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
          best_ms = ms;
          best = A;
        }
      }
      if (m->axis[ax].ch != best.ch) m->bulk_dirty = m->dir_dirty = m->ag_seg_dirty = true;
      m->axis[ax] = best;
    }
    // the slab thickness of the x and y sweeps (0 = whole axes), over whole
    // diffusion steps; slabs up to the size of L2
    build_all(m);
    int l2 = 0;
    BFVM_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, m->device));
    const size_t plane_bytes = (size_t)m->nx * m->ny * m->S * m->elem();
    int best_k = 0;
    float best_ms = 1e30f;
    for (int k : {0, 2, 4, 8, 16, 32, 64}) {
      if (k > 0 && (k >= m->nz || (size_t)k * plane_bytes > (size_t)l2)) continue;
      m->slab_planes = k;
      step_once(m, dt, BFVM_STEP_DIFFUSION, nullptr);  // warm-up
      BFVM_CUDA(cudaEventRecord(e0, m->stream));
      for (int r = 0; r < reps; ++r) step_once(m, dt, BFVM_STEP_DIFFUSION, nullptr);
      BFVM_CUDA(cudaEventRecord(e1, m->stream));
      BFVM_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      BFVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best_ms) {
        best_ms = ms;
        best_k = k;
      }
    }
    m->slab_planes = best_k;
    // whether the bulk and cell updates run inside the x sweep's prologue
    // (same results either way), over whole steps
    if (!m->bulk_vox.empty() || m->n_agents > 0) {
      int best_f = 0;
      best_ms = 1e30f;
      for (int f : {0, 1}) {
        m->fuse_sources = f;
        step_once(m, dt, BFVM_STEP_ALL, nullptr);  // warm-up (and its lists)
        BFVM_CUDA(cudaEventRecord(e0, m->stream));
        for (int r = 0; r < reps; ++r) step_once(m, dt, BFVM_STEP_ALL, nullptr);
        BFVM_CUDA(cudaEventRecord(e1, m->stream));
        BFVM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        BFVM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best_ms) {
          best_ms = ms;
          best_f = f;
        }
      }
      m->fuse_sources = best_f;
    }
  } catch (...) {
    m->fuse_sources = saved_fuse;
    m->slab_planes = saved_slab;
    m->path = saved_path;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemcpyAsync(m->p.ptr, save.ptr, bytes, cudaMemcpyDeviceToDevice, m->stream);
    cudaStreamSynchronize(m->stream);
    save.release();
    throw;
  }
  m->path = saved_path;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BFVM_CUDA(cudaMemcpyAsync(m->p.ptr, save.ptr, bytes, cudaMemcpyDeviceToDevice, m->stream));
  BFVM_CUDA(cudaStreamSynchronize(m->stream));
  save.release();
  build_all(m);
  check_status(m);
}

}  // namespace bfvm_rt

extern "C" {

int bfvm_tune_sweeps(bfvm_solver* m, double dt, int reps) {
  return SOLVER_CALL(m, tune_sweeps(m, dt, reps));
}

int bfvm_get_sweep_kernel(bfvm_solver* m, int axis, int* kind) {
  return SOLVER_CALL(m, {
    require(axis >= 0 && axis < 3 && kind != nullptr, "bad arguments");
    *kind = m->axis[axis].kind;
  });
}

int bfvm_get_sweep_config(bfvm_solver* m, int axis, int* config) {
  return SOLVER_CALL(m, {
    require(axis >= 0 && axis < 3 && config != nullptr, "bad arguments");
    config[0] = m->axis[axis].ch;
    config[1] = m->axis[axis].tw;
    config[2] = m->axis[axis].minb;
    config[3] = m->axis[axis].stages == 3 ? 3 : 2;
  });
}

int bfvm_set_row_build(bfvm_solver* m, int build) {
  return SOLVER_CALL(m, {
    require(build >= 0 && build <= 2, "row build must be 0, 1 or 2");
    m->axis[0].build = build;
  });
}

int bfvm_get_row_build(bfvm_solver* m, int* requested, int* effective) {
  return SOLVER_CALL(m, {
    require(requested != nullptr && effective != nullptr, "bad arguments");
    *requested = m->axis[0].build;
    const RowsPlan P = plan_rows(m);
    *effective = P.ok ? P.build : 0;
  });
}

int bfvm_set_row_stages(bfvm_solver* m, int stages) {
  return SOLVER_CALL(m, {
    require(stages == 2 || stages == 3, "stages must be 2 or 3");
    m->axis[0].stages = stages;
  });
}

int bfvm_synchronize(bfvm_solver* m) {
  return SOLVER_CALL(m, {
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
    wait_transfers(m);
    check_status(m);
  });
}

int bfvm_set_fuse_sources(bfvm_solver* m, int fuse) {
  return SOLVER_CALL(m, { m->fuse_sources = fuse ? 1 : 0; });
}

int bfvm_get_fuse_sources(bfvm_solver* m, int* fuse) {
  return SOLVER_CALL(m, {
    require(fuse != nullptr, "null output pointer");
    *fuse = m->fuse_sources;
  });
}

int bfvm_set_kernel_path(bfvm_solver* m, int path) {
  return SOLVER_CALL(m, {
    require(path >= BFVM_PATH_AUTO && path <= BFVM_PATH_DIRECT, "unknown kernel path");
    m->path = path;
  });
}

int bfvm_get_stream(bfvm_solver* m, void** stream) {
  return SOLVER_CALL(m, {
    require(stream != nullptr, "null output pointer");
    *stream = (void*)m->stream;
  });
}

int bfvm_get_launch_count(bfvm_solver* m, int64_t* count) {
  return SOLVER_CALL(m, {
    require(count != nullptr, "null output pointer");
    *count = m->launches;
  });
}

int bfvm_profile_step(bfvm_solver* m, double dt, int nsteps, int flags, double* ms) {
  return SOLVER_CALL(m, {
    require(ms != nullptr && nsteps > 0, "bad arguments");
    require(flags & BFVM_STEP_DIFFUSION, "profiling needs the diffusion sweeps");
    cudaEvent_t ev[5];
    for (auto& e : ev) BFVM_CUDA(cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0};
    for (int it = 0; it < nsteps; ++it) {
      step_once(m, dt, flags, ev);
      BFVM_CUDA(cudaEventSynchronize(ev[4]));
      for (int a = 0; a < 4; ++a) {
        float t = 0;
        BFVM_CUDA(cudaEventElapsedTime(&t, ev[a], ev[a + 1]));
        acc[a] += t;
      }
    }
    for (int a = 0; a < 4; ++a) ms[a] = acc[a] / nsteps;
    for (auto& e : ev) cudaEventDestroy(e);
    check_status(m);
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Gather without allocation.
//
// bfvm_get_voxel_densities allocates two small device buffers per call (the
// voxel list and the gathered values).  Some callers can't call cudaMalloc:
// cudaMalloc and cudaFree can synchronise the whole device, which a host loop
// that must not stall cannot afford, and in a process whose device memory is
// held by another allocator (a framework's caching allocator) a fresh
// cudaMalloc may fail.  bfvm_get_voxel_densities_noalloc does the same gather
// through one file-scope device array of fixed size instead.  Every GPU that
// loads the library holds the array until the process exits; every call (on
// any solver of that device) reuses it and it keeps the last call's contents.
// Nothing in it needs to start at zero: the voxel list and the values are
// written before they are read.  Calls whose GPU work overlaps (from several
// host threads, or on several solvers' streams at once) race on the array;
// each call synchronises its solver's stream before returning, so calls made
// one after another never overlap.

namespace {

constexpr size_t kGatherScratchBytes = (size_t)4 << 20;  // 4 MiB
__device__ __align__(256) unsigned char g_gather_scratch[kGatherScratchBytes];

std::mutex g_gather_scratch_mutex;
void* g_gather_scratch_addr[64] = {};  // per device, set on first use

// Device address of g_gather_scratch on the current device (the caller has
// made m->device current).  In host code the array's name is only a host-side
// stand-in, so the address is looked up once per device.
void* gather_scratch(int device) {
  require(device >= 0 && device < 64, "device index out of range for the static scratch");
  std::lock_guard<std::mutex> g(g_gather_scratch_mutex);
  if (g_gather_scratch_addr[device] == nullptr) {
    void* ptr = nullptr;
    BFVM_CUDA(cudaGetSymbolAddress(&ptr, g_gather_scratch));
    require(ptr != nullptr, "cudaGetSymbolAddress returned no address", BFVM_ERR_CUDA);
    g_gather_scratch_addr[device] = ptr;
  }
  return g_gather_scratch_addr[device];
}

}  // namespace

extern "C" int bfvm_get_voxel_densities_noalloc(bfvm_solver* m, int64_t count,
                                                const int64_t* voxels, double* values) {
  return SOLVER_CALL(m, {
    require(count >= 0 && (count == 0 || (voxels && values)), "bad arguments");
    // bound count before any product of it, so no size below wraps around
    const size_t per_voxel = sizeof(int64_t) + (size_t)std::max(m->S, 1) * sizeof(double);
    require((uint64_t)count <= kGatherScratchBytes / per_voxel,
            "bfvm_get_voxel_densities_noalloc: " + std::to_string(count) + " voxels x " +
                std::to_string(m->S) + " densities do not fit the " +
                std::to_string(kGatherScratchBytes) +
                "-byte static scratch (at most count*(8 + 8*S) bytes)");
    const size_t vox_bytes = ((size_t)count * sizeof(int64_t) + 255) & ~(size_t)255;
    const size_t val_bytes = (size_t)count * m->S * sizeof(double);
    require(vox_bytes + val_bytes <= kGatherScratchBytes,
            "bfvm_get_voxel_densities_noalloc: " + std::to_string(count) + " voxels x " +
                std::to_string(m->S) + " densities need " +
                std::to_string(vox_bytes + val_bytes) + " bytes of the " +
                std::to_string(kGatherScratchBytes) +
                "-byte static scratch (at most count*(8 + 8*S) bytes, after rounding the "
                "voxel list up to 256 bytes)");
    validate_voxels(m, count, voxels);
    if (count == 0) return;
    unsigned char* base = static_cast<unsigned char*>(gather_scratch(m->device));
    int64_t* d_vox = reinterpret_cast<int64_t*>(base);
    double* d_out = reinterpret_cast<double*>(base + vox_bytes);
    BFVM_CUDA(cudaMemcpyAsync(d_vox, voxels, (size_t)count * sizeof(int64_t),
                              cudaMemcpyHostToDevice, m->stream));
    if (m->precision == BFVM_FP64)
      gather<double>(m, count, d_vox, d_out);
    else
      gather<float>(m, count, d_vox, d_out);
    BFVM_CUDA(cudaMemcpyAsync(values, d_out, val_bytes, cudaMemcpyDeviceToHost, m->stream));
    BFVM_CUDA(cudaStreamSynchronize(m->stream));
  });
}
