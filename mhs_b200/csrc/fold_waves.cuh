// The fold as a planned multi-kernel pipeline (mhs/kernels/fold.py:
// 290-367): the Boussinesq correction of every band pair -- a source that
// reaches the surface seen from a receiver in its band -- is the weighted
// sum, over the receiver's polar grid on z = 0, of the point-load response
// times the element's surface load there minus the load at the receiver's
// foot.  Each stage runs as its own kernel, so each gets the registers and
// occupancy its own arithmetic needs:
//
//   plan     per pair: radial breaks and angular rules -> panels and nodes
//            (counts, then prefix sums); the host reads the totals back
//   foot     per pair: the surface load at the receiver's foot
//   nodes    per panel: node positions and weights; each node classified as
//            a far node (12 x 12 or 8 x 8 rule) or a near node keyed by the
//            forms of its three edges (how many take the small-|u| and the
//            large-|u| series), so that every warp of the load kernels runs
//            one code path
//   scatter  stable-enough class lists (order inside a list does not enter
//            any sum: loads are stored per node)
//   far/near the surface loads, one thread per node
//   accum    per pair, panel by panel in grid order: the weighted
//            point-load products of each panel reduced in a fixed tree
//            order and added to the pair's running sum, so the result does
//            not depend on how panels were grouped into waves
//   finish   per pair: the disk term and the add into the pair's table row
//
// Nodes live in bounded waves of whole panels (the workspace's fold
// region), pairs in batches; both sizes come from the totals read back
// after the plan, one short stream synchronisation per batch.
#pragma once

namespace fold_waves {

constexpr int NCLS = 12;          // 10 near signatures, far 12 x 12, far 8 x 8

constexpr int CLS_FAR12 = 10;
constexpr int CLS_FAR8 = 11;

// Near signature of a node from its edge-form counts (n_small, n_large),
// n_small + n_large <= 3; the inverse tables give the counts back.
MHS_FI int near_sig(int ns, int nl) {
  // rows ns = 0..3, columns nl = 0..3 (entries with ns + nl > 3 unused)
  const int base[4] = {0, 4, 7, 9};
  return base[ns] + nl;
}
__device__ const int kSigSmall[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
__device__ const int kSigLarge[10] = {0, 1, 2, 3, 0, 1, 2, 0, 1, 0};

// Device-side counters shared by the fold kernels of one request chunk.
struct Hdr {
  long long n_st, n_pairs;               // straddling sources, band pairs (chunk)
  long long q_batch, n_batch, max_panel; // panels, nodes, largest panel (batch)
  long long wave_q0, wave_q1;            // panels of the current wave
  long long wave_n0, wave_nodes;         // first node and node count of the wave
  long long cls_off[NCLS + 1];           // class offsets in the list array
  int cls_count[NCLS];
  int cls_fill[NCLS];
};

// Per straddling source: far rules (double, and float for the mixed form)
// and the sigma_zz row of the surface load.
template <int P, class RF>
struct Src {
  SmemRules<P> rd;
  std::conditional_t<std::is_same<RF, float>::value, FloatRules<P>, NoRules> fr;
  SurfaceLoadConsts slc;
};

// ------------------------------------------------------------- band scan
// One block: straddle ranks, their sources and the prefix of band pairs by
// straddle rank; totals into the header.
__global__ void __launch_bounds__(1024)
k_band_scan(int64_t n_src, const SrcPrep* __restrict__ prep, const int* __restrict__ cnt,
            int* __restrict__ st_rank, int* __restrict__ st_src, long long* __restrict__ st_off,
            Hdr* __restrict__ hdr) {
  __shared__ long long s_pairs[1024];
  __shared__ int s_st[1024];
  __shared__ long long base_pairs;
  __shared__ int base_st;
  if (threadIdx.x == 0) {
    base_pairs = 0;
    base_st = 0;
  }
  __syncthreads();
  for (int64_t s0 = 0; s0 < n_src; s0 += 1024) {
    const int64_t s = s0 + threadIdx.x;
    const int is_st = (s < n_src && prep[s].straddle) ? 1 : 0;
    const long long np = is_st ? (long long)cnt[s] : 0;
    s_st[threadIdx.x] = is_st;
    s_pairs[threadIdx.x] = np;
    __syncthreads();
    // inclusive Hillis-Steele scans
    for (int d = 1; d < 1024; d <<= 1) {
      const int a = threadIdx.x >= d ? s_st[threadIdx.x - d] : 0;
      const long long b = threadIdx.x >= d ? s_pairs[threadIdx.x - d] : 0;
      __syncthreads();
      s_st[threadIdx.x] += a;
      s_pairs[threadIdx.x] += b;
      __syncthreads();
    }
    if (s < n_src) {
      const int rank = base_st + s_st[threadIdx.x] - is_st;
      st_rank[s] = is_st ? rank : -1;
      if (is_st) {
        st_src[rank] = (int)s;
        st_off[rank] = base_pairs + s_pairs[threadIdx.x] - np;
      }
    }
    __syncthreads();
    if (threadIdx.x == 1023) {
      base_st += s_st[1023];
      base_pairs += s_pairs[1023];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st_off[base_st] = base_pairs;
    hdr->n_st = base_st;
    hdr->n_pairs = base_pairs;
  }
}

// ----------------------------------------------------------- source data
template <int P, int KC, class RF>
__global__ void __launch_bounds__(128)
k_src(int j0, int nj, const int* __restrict__ st_src, const SrcPrep* __restrict__ prep, double mu,
      double lam, Src<P, RF>* __restrict__ out) {
  const int j = blockIdx.x;
  if (j >= nj) return;
  const SrcPrep& sp = prep[st_src[j0 + j]];
  Src<P, RF>& d = out[j];
  const Material m = make_material(mu, lam);
  d.rd.build(sp.f, threadIdx.x, blockDim.x);
  if (threadIdx.x < NLIFT) {
    double col[3] = {};
    szz_coefficient(sp.f, sp.eps, m, threadIdx.x, col);
    for (int c = 0; c < 3; ++c) d.slc.coef[c][threadIdx.x] = col[c];
  }
  if (threadIdx.x == NLIFT) surface_load_ezz(sp.f, sp.eps, m, d.slc);
  if constexpr (std::is_same<RF, float>::value) build_float_rules<P>(sp.f, d.fr, threadIdx.x, blockDim.x);
}

// ------------------------------------------------------------- the plan
// Straddle rank of global pair p (st_off ascending, st_off[j] <= p).
__device__ __forceinline__ int pair_straddler(const long long* st_off, int n_st, long long p) {
  int lo = 0, hi = n_st - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (st_off[mid] <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct PairGeom {
  FoldPair fp;
  double diam;
};

__device__ __forceinline__ void pair_geom(const double* obs, int64_t lo, int oc, const SrcPrep& sp,
                                          FoldPair& fp) {
  const int64_t o = lo + oc;
  const double x[3] = {obs[3 * o], obs[3 * o + 1], obs[3 * o + 2]};
  fold_pair_setup(x, sp.centre, sp.r_f, sp.eps, fp);
}

// Panels and nodes of each pair of the batch [p0, p0 + np): band pair ->
// (straddler, receiver), breaks, kept panels and their angular rules.  One
// thread per pair; the largest panel's node count goes to hdr->max_panel.
__global__ void __launch_bounds__(128)
k_pairs(long long p0, int np, int64_t lo, int64_t n_chunk, const double* __restrict__ obs,
        const SrcPrep* __restrict__ prep, const int* __restrict__ list,
        const int* __restrict__ st_src, const long long* __restrict__ st_off,
        Hdr* __restrict__ hdr, int* __restrict__ pair_st, int* __restrict__ pair_oc,
        long long* __restrict__ pair_npanel, long long* __restrict__ pair_nnode,
        int* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const long long p = p0 + i;
  const int j = pair_straddler(st_off, (int)hdr->n_st, p);
  const int s = st_src[j];
  const int oc = list[(int64_t)s * n_chunk + (p - st_off[j])];
  pair_st[i] = j;
  pair_oc[i] = oc;
  const SrcPrep& sp = prep[s];
  FoldPair fp;
  pair_geom(obs, lo, oc, sp, fp);
  double br[FOLD_MAX_BREAKS];
  double R1;
  const int nb = fold_breaks(fp.rho_s, fp.zeta, sp.r_f, sp.eps, sp.diam, br, &R1);
  long long npan = 0, nnode = 0, big = 0;
  if (nb < 0) {
    atomicOr(status, MHS_DEV_FOLD_GRID_OVERFLOW);
  } else {
    for (int k = 0; k + 1 < nb; ++k) {
      if (br[k + 1] - br[k] < 1e-9 * sp.eps) continue;
      AngRule A;
      fold_panel_rule(fp, br[k], br[k + 1], A);
      ++npan;
      if (A.n < 0) {
        atomicOr(status, MHS_DEV_FOLD_GRID_OVERFLOW);
        continue;
      }
      const long long n = (long long)cst::FOLD_N_RADIAL * A.n;
      nnode += n;
      big = n > big ? n : big;
    }
  }
  pair_npanel[i] = npan;
  pair_nnode[i] = nnode;
  if (big) atomicMax(reinterpret_cast<unsigned long long*>(&hdr->max_panel), (unsigned long long)big);
}

// Exclusive prefix sum in place over a[0..n) (a[n] receives the total),
// one block; optionally the maximum of the inputs into *mx.
__global__ void __launch_bounds__(1024)
k_scan(long long* __restrict__ a, long long n, long long* __restrict__ total,
       long long* __restrict__ mx) {
  __shared__ long long sh[1024];
  __shared__ long long base, best;
  if (threadIdx.x == 0) {
    base = 0;
    best = 0;
  }
  __syncthreads();
  for (long long i0 = 0; i0 < n; i0 += 1024) {
    const long long i = i0 + threadIdx.x;
    const long long v = i < n ? a[i] : 0;
    sh[threadIdx.x] = v;
    if (mx && v > 0) atomicMax(reinterpret_cast<unsigned long long*>(&best), (unsigned long long)v);
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
      const long long t = threadIdx.x >= d ? sh[threadIdx.x - d] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n) a[i] = base + sh[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) base += sh[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a[n] = base;
    if (total) *total = base;
    if (mx) *mx = best;
  }
}

// Radial interval and first node of every kept panel (one thread per pair;
// the pair's panels start at pair_poff[i], its nodes at pair_noff[i]).
__global__ void __launch_bounds__(128)
k_panels(int np, int64_t lo, const double* __restrict__ obs, const SrcPrep* __restrict__ prep,
         const int* __restrict__ st_src, const int* __restrict__ pair_st,
         const int* __restrict__ pair_oc, const long long* __restrict__ pair_poff,
         const long long* __restrict__ pair_noff, double* __restrict__ pan_ra,
         double* __restrict__ pan_rb, long long* __restrict__ pan_noff,
         int* __restrict__ pan_pair) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > np) return;
  if (i == np) {  // closing entry: the batch's node total
    pan_noff[pair_poff[np]] = pair_noff[np];
    return;
  }
  const SrcPrep& sp = prep[st_src[pair_st[i]]];
  FoldPair fp;
  pair_geom(obs, lo, pair_oc[i], sp, fp);
  double br[FOLD_MAX_BREAKS];
  double R1;
  const int nb = fold_breaks(fp.rho_s, fp.zeta, sp.r_f, sp.eps, sp.diam, br, &R1);
  long long q = pair_poff[i], u = pair_noff[i];
  for (int k = 0; k + 1 < nb; ++k) {
    const double ra = br[k], rb = br[k + 1];
    if (rb - ra < 1e-9 * sp.eps) continue;
    AngRule A;
    fold_panel_rule(fp, ra, rb, A);
    pan_ra[q] = ra;
    pan_rb[q] = rb;
    pan_noff[q] = u;
    pan_pair[q] = i;
    u += A.n < 0 ? 0 : (long long)cst::FOLD_N_RADIAL * A.n;
    ++q;
  }
}

// Surface load at each receiver's foot (one thread per pair).
template <int P, int KC, class RF>
__global__ void __launch_bounds__(128)
k_foot(int np, int j0, int64_t lo, const double* __restrict__ obs,
       const SrcPrep* __restrict__ prep, const int* __restrict__ st_src,
       const int* __restrict__ pair_st, const int* __restrict__ pair_oc,
       const Src<P, RF>* __restrict__ srcs, double* __restrict__ foot) {
  constexpr int NJ = 3 * n_nodes(P);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int j = pair_st[i];
  const SrcPrep& sp = prep[st_src[j]];
  const Src<P, RF>& d = srcs[j - j0];
  const int64_t o = lo + pair_oc[i];
  double sl[NJ] = {};
  fold_surface_load_fast<P, RF>(sp.f, d.rd.r12(), d.rd.r8(), d.slc, obs[3 * o], obs[3 * o + 1],
                                sp.eps, sl);
  for (int jj = 0; jj < NJ; ++jj) foot[(size_t)i * NJ + jj] = sl[jj];
}

// --------------------------------------------------------------- a wave
// Panels [q0, q1) of the batch whose first node lies in
// [w * span, (w + 1) * span); the first node of the wave and its count.
__global__ void k_wave_begin(long long w, long long span, long long nq,
                             const long long* __restrict__ pan_noff, Hdr* __restrict__ hdr) {
  auto first_at = [&](long long v) {  // first panel q with pan_noff[q] >= v
    long long a = 0, b = nq;
    while (a < b) {
      const long long m = (a + b) >> 1;
      if (pan_noff[m] < v) a = m + 1;
      else b = m;
    }
    return a;
  };
  const long long q0 = first_at(w * span), q1 = first_at((w + 1) * span);
  hdr->wave_q0 = q0;
  hdr->wave_q1 = q1;
  hdr->wave_n0 = pan_noff[q0];
  hdr->wave_nodes = pan_noff[q1] - pan_noff[q0];
  for (int c = 0; c < NCLS; ++c) {
    hdr->cls_count[c] = 0;
    hdr->cls_fill[c] = 0;
  }
}

// Edge-form counts (small-|u| series, large-|u| series) of a near node, in
// float: the counts only group nodes into warp-uniform lists -- k_near
// recomputes every edge's form in double -- so a node whose float test lands
// on the other side of a form threshold costs some divergence, not accuracy.
MHS_FI void near_signature_f(const Frame& f, double px, double py, double eps, int& ns, int& nl) {
  const float d0 = (float)(px - f.c[0]), d1 = (float)(py - f.c[1]), d2 = (float)(0.0 - f.c[2]);
  const float z = d0 * (float)f.n[0] + d1 * (float)f.n[1] + d2 * (float)f.n[2];
  const float X0 = d0 * (float)f.e1[0] + d1 * (float)f.e1[1] + d2 * (float)f.e1[2];
  const float X1 = d0 * (float)f.e2[0] + d1 * (float)f.e2[1] + d2 * (float)f.e2[2];
  const float h2 = z * z + (float)(eps * eps);
  float pr[3][2];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    pr[k][0] = (float)f.p[k][0] - X0;
    pr[k][1] = (float)f.p[k][1] - X1;
  }
  const float s2 = (float)cst::SMALL_U_OVER_RHO_SQ, l2 = (float)cst::SERIES_U_OVER_RHO_SQ;
  ns = 0;
  nl = 0;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int e2 = e == 2 ? 0 : e + 1;
    const float ev0 = pr[e2][0] - pr[e][0], ev1 = pr[e2][1] - pr[e][1];
    const float iL = rsqrtf(ev0 * ev0 + ev1 * ev1);
    const float s1 = ev0 * iL, sy = ev1 * iL;
    const float dp = pr[e][0] * sy - pr[e][1] * s1;
    const float ua = pr[e][0] * s1 + pr[e][1] * sy, ub = pr[e2][0] * s1 + pr[e2][1] * sy;
    const float rho2 = dp * dp + h2;
    const float a2 = ua * ua, b2 = ub * ub;
    const float umax2 = a2 > b2 ? a2 : b2, umin2 = a2 < b2 ? a2 : b2;
    if (umax2 <= s2 * rho2) ++ns;
    else if (ua * ub > 0.0f && umin2 >= l2 * rho2) ++nl;
  }
}

// Nodes of the wave's panels: position, weight, pair, class.  One warp per
// panel (grid-stride over the wave's panels): each lane takes angular nodes
// j (one sincos each) and writes the panel's six radial nodes at j, in the
// grid's order ir * n_ang + j.
// Three blocks of 256 per SM (80 registers, a few spills): 1.7 ms less per
// config-2 step than two at 128 registers; the kernel is latency-bound.
constexpr int NODES_MIN_BLOCKS = 3;

template <int P>
__global__ void __launch_bounds__(256, NODES_MIN_BLOCKS)
k_nodes(double near_l, int np, int64_t lo, const double* __restrict__ obs,
        const SrcPrep* __restrict__ prep, const int* __restrict__ st_src,
        const int* __restrict__ pair_st, const int* __restrict__ pair_oc,
        const int* __restrict__ pan_pair, const double* __restrict__ pan_ra,
        const double* __restrict__ pan_rb, const long long* __restrict__ pan_noff,
        const Hdr* __restrict__ hdr, double* __restrict__ npx, double* __restrict__ npy,
        double* __restrict__ nw, int* __restrict__ npair, unsigned char* __restrict__ ncls) {
  constexpr int NR = cst::FOLD_N_RADIAL;
  __shared__ AngRule sA[8];
  __shared__ FoldPair sfp[8];
  __shared__ int spair[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long q0 = hdr->wave_q0, q1 = hdr->wave_q1, n0 = hdr->wave_n0;
  const double* gx6 = d_glx + gl_offset(NR);
  const double* gw6 = d_glw + gl_offset(NR);
  const double* gx4 = d_glx + gl_offset(cst::FOLD_N_ANGULAR);
  const double* gw4 = d_glw + gl_offset(cst::FOLD_N_ANGULAR);
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long q = q0 + (long long)blockIdx.x * (blockDim.x >> 5) + wid; q < q1; q += nwarps) {
    if (lane == 0) {
      const int i = pan_pair[q];
      const SrcPrep& sp = prep[st_src[pair_st[i]]];
      FoldPair f;
      pair_geom(obs, lo, pair_oc[i], sp, f);
      fold_panel_rule(f, pan_ra[q], pan_rb[q], sA[wid]);
      sfp[wid] = f;
      spair[wid] = i;
    }
    __syncwarp();
    const AngRule& A = sA[wid];
    const FoldPair& fp = sfp[wid];
    const int i = spair[wid];
    const SrcPrep& sp = prep[st_src[pair_st[i]]];
    const double ra = pan_ra[q], rb = pan_rb[q];
    const int na = A.n > 0 ? A.n : 0;
    const long long base = pan_noff[q] - n0;
    double R[NR], wr[NR];
#pragma unroll
    for (int ir = 0; ir < NR; ++ir) {
      R[ir] = ra + (rb - ra) * (0.5 * (gx6[ir] + 1.0));
      wr[ir] = (rb - ra) * (0.5 * gw6[ir]);
    }
    for (int jn = lane; jn < na; jn += 32) {
      double th, wt;
      fold_ang_node(A, gx4, gw4, jn, &th, &wt);
      double sn, cs;
      sincos(th, &sn, &cs);
#pragma unroll
      for (int ir = 0; ir < NR; ++ir) {
        const double px = fp.xh0 + R[ir] * cs, py = fp.xh1 + R[ir] * sn;
        int cls = surface_class(sp.f, px, py, sp.eps);
        if (cls == SL_NEAR && near_l < cst::D_STAR) {
          // the mixed form: closed form only within near_l element lengths
          const double d0 = px - sp.f.c[0], d1 = py - sp.f.c[1], d2 = 0.0 - sp.f.c[2];
          const double D = sqrt(((d0 * d0 + d1 * d1) + d2 * d2) + sp.eps * sp.eps);
          if (D > near_l * sp.f.L) cls = SL_FAR12;
        }
        if (cls == SL_NEAR) {
          int ns, nl;
          near_signature_f(sp.f, px, py, sp.eps, ns, nl);
          cls = near_sig(ns, nl);
        } else {
          cls = cls == SL_FAR8 ? CLS_FAR8 : CLS_FAR12;
        }
        const long long u = base + (long long)ir * na + jn;
        npx[u] = px;
        npy[u] = py;
        nw[u] = wr[ir] * wt * R[ir];
        npair[u] = i;
        ncls[u] = (unsigned char)cls;
      }
    }
    __syncwarp();
  }
}

// Class counts of the wave's nodes (block-aggregated: one global add per
// class per block tile).
constexpr int SCAT_PER_THREAD = 4;

__global__ void __launch_bounds__(256)
k_count(Hdr* __restrict__ hdr, const unsigned char* __restrict__ ncls) {
  __shared__ int s_cnt[NCLS];
  const long long n = hdr->wave_nodes;
  const long long tile = (long long)blockDim.x * SCAT_PER_THREAD;
  if (threadIdx.x < NCLS) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  for (long long t0 = (long long)blockIdx.x * tile; t0 < n; t0 += (long long)gridDim.x * tile) {
#pragma unroll
    for (int k = 0; k < SCAT_PER_THREAD; ++k) {
      const long long u = t0 + (long long)k * blockDim.x + threadIdx.x;
      const int cls = u < n ? ncls[u] : -1;
      // lanes of one class: the lowest adds their count
      const unsigned m = __match_any_sync(0xffffffffu, cls);
      if (cls >= 0 && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(&s_cnt[cls], __popc(m));
    }
  }
  __syncthreads();
  if (threadIdx.x < NCLS && s_cnt[threadIdx.x]) atomicAdd(&hdr->cls_count[threadIdx.x], s_cnt[threadIdx.x]);
}

// Class offsets of the wave (and the census of its nodes and near edges).
__global__ void k_wave_classes(Hdr* __restrict__ hdr, unsigned long long* __restrict__ census) {
  long long off = 0;
  for (int c = 0; c < NCLS; ++c) {
    hdr->cls_off[c] = off;
    off += hdr->cls_count[c];
  }
  hdr->cls_off[NCLS] = off;
  if (census) {
    unsigned long long near = 0, es = 0, el = 0, ec = 0;
    for (int c = 0; c < 10; ++c) {
      const unsigned long long n = (unsigned long long)hdr->cls_count[c];
      near += n;
      es += n * kSigSmall[c];
      el += n * kSigLarge[c];
      ec += n * (3 - kSigSmall[c] - kSigLarge[c]);
    }
    census[MHS_CENSUS_NEAR] += near;
    census[MHS_CENSUS_FAR12] += (unsigned long long)hdr->cls_count[CLS_FAR12];
    census[MHS_CENSUS_FAR8] += (unsigned long long)hdr->cls_count[CLS_FAR8];
    census[MHS_CENSUS_EDGE_CLOSED] += ec;
    census[MHS_CENSUS_EDGE_SMALL] += es;
    census[MHS_CENSUS_EDGE_LARGE] += el;
  }
}

// Node indices into their class lists: per block tile of
// SCAT_PER_THREAD x blockDim nodes, the warps' class counts are combined in
// shared memory and each class takes one global add per tile.
__global__ void __launch_bounds__(256)
k_scatter(Hdr* __restrict__ hdr, const unsigned char* __restrict__ ncls, int* __restrict__ nlist) {
  constexpr int WMAX = 8;
  __shared__ int w_cnt[SCAT_PER_THREAD][WMAX][NCLS];
  __shared__ int b_base[NCLS];
  const long long n = hdr->wave_nodes;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long tile = (long long)blockDim.x * SCAT_PER_THREAD;
  for (long long t0 = (long long)blockIdx.x * tile; t0 < n; t0 += (long long)gridDim.x * tile) {
    int cls[SCAT_PER_THREAD];
    unsigned mk[SCAT_PER_THREAD];
#pragma unroll
    for (int k = 0; k < SCAT_PER_THREAD; ++k) {
      const long long u = t0 + (long long)k * blockDim.x + threadIdx.x;
      cls[k] = u < n ? ncls[u] : -1;
      mk[k] = 0;
    }
    // per warp, per sub-tile: count of each class, and this lane's peers
#pragma unroll
    for (int k = 0; k < SCAT_PER_THREAD; ++k) {
      if (lane < NCLS) w_cnt[k][wid][lane] = 0;
      mk[k] = __match_any_sync(0xffffffffu, cls[k]);
      __syncwarp();
      if (cls[k] >= 0 && lane == __ffs(mk[k]) - 1) w_cnt[k][wid][cls[k]] = __popc(mk[k]);
    }
    __syncthreads();
    // per class, the counts become exclusive prefixes in (sub-tile, warp)
    // order, and the block's run of the class list is claimed
    if (threadIdx.x < NCLS) {
      const int c = threadIdx.x;
      int tot = 0;
      for (int k = 0; k < SCAT_PER_THREAD; ++k)
        for (int w = 0; w < nw; ++w) {
          const int v = w_cnt[k][w][c];
          w_cnt[k][w][c] = tot;
          tot += v;
        }
      b_base[c] = tot ? atomicAdd(&hdr->cls_fill[c], tot) : 0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAT_PER_THREAD; ++k) {
      const int c = cls[k];
      if (c >= 0) {
        const int off = b_base[c] + w_cnt[k][wid][c] + __popc(mk[k] & ((1u << lane) - 1u));
        const long long u = t0 + (long long)k * blockDim.x + threadIdx.x;
        nlist[hdr->cls_off[c] + off] = (int)u;
      }
    }
    __syncthreads();
  }
}

// Far loads: one thread per node of the far lists.  The FP64 form takes
// mhs's rules (12 x 12; 8 x 8 for the far-8 class, beyond D_STAR_DISTANT L);
// the mixed form takes its float MIXED_GAUSS_N_FAR rule for both classes (every
// far node lies beyond D_STAR L).
template <int P, int KC, class RF>
__device__ __forceinline__ QuadRuleT<RF> far_rule(const Src<P, RF>& d, bool r8) {
  if constexpr (std::is_same<RF, float>::value) {
    return float_rule_far<P>(d.fr);
  } else {
    constexpr int K = n_nodes(P), N12 = cst::FAR_GAUSS_N * cst::FAR_GAUSS_N;
    constexpr int N8 = cst::FAR_GAUSS_N_DISTANT * cst::FAR_GAUSS_N_DISTANT;
    const int off = r8 ? N12 : 0;
    return QuadRuleT<double>{r8 ? N8 : N12, d.rd.e0 + off, d.rd.e1 + off, d.rd.wq + off,
                             d.rd.Nq + off * K};
  }
}

// Launch bounds of the load and accumulation kernels at P0, from timing them
// on config 2 (FP64): k_far at 5 blocks of 128 per SM (96 registers; asking
// for one block lets it take 248 and runs 30 % slower), k_near at 5 (96
// registers, 10 % faster than 4 despite a few spills), k_accum at 5 (96
// registers, with the next node's loads in flight: 33 % faster than its
// unbounded 132 registers without the prefetch).  P1 and P2 keep their
// registers (bounding them spills).
constexpr int FAR_MIN_BLOCKS = 5;
constexpr int NEAR_MIN_BLOCKS_P0 = 5;
constexpr int ACCUM_MIN_BLOCKS = 5;

template <int P, int KC, class RF>
__global__ void __launch_bounds__(128, P == 0 ? FAR_MIN_BLOCKS : 1)
k_far(const Hdr* __restrict__ hdr, const int* __restrict__ nlist, const double* __restrict__ npx,
      const double* __restrict__ npy, const int* __restrict__ npair,
      const int* __restrict__ pair_st, int j0, const int* __restrict__ st_src,
      const SrcPrep* __restrict__ prep, const Src<P, RF>* __restrict__ srcs,
      double* __restrict__ load, long long cap) {
  constexpr int K = n_nodes(P);
  constexpr int NJ = 3 * K;
  const long long a = hdr->cls_off[CLS_FAR12], b = hdr->cls_off[CLS_FAR8 + 1];
  const long long r8_from = hdr->cls_off[CLS_FAR8];
  for (long long e = a + (long long)blockIdx.x * blockDim.x + threadIdx.x; e < b;
       e += (long long)gridDim.x * blockDim.x) {
    const int u = nlist[e];
    const int j = pair_st[npair[u]];
    const SrcPrep& sp = prep[st_src[j]];
    const Src<P, RF>& d = srcs[j - j0];
    const double xx[3] = {npx[u], npy[u], 0.0};
    double z, X0, X1;
    to_plane(sp.f, xx, z, X0, X1);
    const double h2 = z * z + sp.eps * sp.eps;
    double sl[NJ] = {};
    surface_load_far<P, RF>(far_rule<P, KC, RF>(d, e >= r8_from), d.slc, z, X0, X1, h2, sl);
#pragma unroll
    for (int jj = 0; jj < NJ; ++jj) load[(size_t)jj * cap + u] = sl[jj];
  }
}

// Near loads: one thread per node of the near lists.  Every node of one
// list has the same number of small-|u| and large-|u| edges, so a warp
// (away from list boundaries) takes one path through the edge forms: its
// edges are visited small-series ones first, then large-series ones, then
// closed-form ones.
template <int P, int KC>
__global__ void __launch_bounds__(128, P == 0 ? NEAR_MIN_BLOCKS_P0 : 1)
k_near(const Hdr* __restrict__ hdr, const int* __restrict__ nlist, const double* __restrict__ npx,
       const double* __restrict__ npy, const int* __restrict__ npair,
       const int* __restrict__ pair_st, int j0, const int* __restrict__ st_src,
       const SrcPrep* __restrict__ prep, const SurfaceLoadConsts* __restrict__ slcs,
       long long slc_stride, double* __restrict__ load, long long cap) {
  using S = SurfaceSpec<P>;
  constexpr Spec spc = S::spec;
  constexpr int K = n_nodes(P);
  constexpr int NJ = 3 * K;
  constexpr int NB = spc.b_off[MS] > 0 ? spc.b_off[MS] : 1;
  const long long a = hdr->cls_off[0], b = hdr->cls_off[10];
  for (long long e = a + (long long)blockIdx.x * blockDim.x + threadIdx.x; e < b;
       e += (long long)gridDim.x * blockDim.x) {
    const int u = nlist[e];
    const int j = pair_st[npair[u]];
    const SrcPrep& sp = prep[st_src[j]];
    const SurfaceLoadConsts& c =
        *reinterpret_cast<const SurfaceLoadConsts*>(reinterpret_cast<const char*>(slcs) +
                                                    (size_t)(j - j0) * slc_stride);
    const double eps = sp.eps;
    const double xx[3] = {npx[u], npy[u], 0.0};
    double z, X0, X1;
    to_plane(sp.f, xx, z, X0, X1);
    const double h2 = z * z + eps * eps;
    double pr[3][2];
    foot_vertices(sp.f, X0, X1, pr);
    // edge slots ordered small-series, large-series, closed; the form of
    // position i depends only on the node's list, so it is warp-uniform
    EdgeGeom g[3];
    int form[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      g[k] = edge_geom_rcp(pr, k, h2);
      form[k] = edge_regime_sq(g[k].ua, g[k].ub, g[k].rho2);
    }
    int order[3] = {0, 0, 0}, no = 0;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const int want = f == 0 ? EDGE_SMALL : (f == 1 ? EDGE_LARGE : EDGE_CLOSED);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const bool hit = form[k] == want;
        // branch-free append: positions 0..2 as selects
        order[0] = (hit && no == 0) ? k : order[0];
        order[1] = (hit && no == 1) ? k : order[1];
        order[2] = (hit && no == 2) ? k : order[2];
        no += hit ? 1 : 0;
      }
    }
    const int ns = (form[0] == EDGE_SMALL) + (form[1] == EDGE_SMALL) + (form[2] == EDGE_SMALL);
    const int nl = (form[0] == EDGE_LARGE) + (form[1] == EDGE_LARGE) + (form[2] == EDGE_LARGE);
    double BN1[NB], BN2[NB], BD[MS];
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      BN1[t] = 0.0;
      BN2[t] = 0.0;
    }
#pragma unroll
    for (int t = 0; t < MS; ++t) BD[t] = 0.0;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
      const int k = i == 0 ? order[0] : (i == 1 ? order[1] : order[2]);
      const EdgeGeom ge = k == 0 ? g[0] : (k == 1 ? g[1] : g[2]);
      double Pt[MS][8];
      if (i < ns) edge_small<S>(ge.ua, ge.ub, sqrt(ge.rho2), Pt);
      else if (i < ns + nl) edge_large<S>(ge.ua, ge.ub, ge.rho2, Pt);
      else edge_closed<S, true>(ge.ua, ge.ub, ge.rho2, Pt);
      edge_accumulate<S>(ge, Pt, BN1, BN2, BD);
    }
    MomentTable<S> T;
    closed_finish_t<S, true>(pr, h2, BN1, BN2, BD, T);
    double sl[NJ] = {};
    surface_load_near<P>(sp.f, T, c, z, X0, X1, sl);
#pragma unroll
    for (int jj = 0; jj < NJ; ++jj) load[(size_t)jj * cap + u] = sl[jj];
  }
}

// Accumulation: per panel, the weighted point-load products of its nodes
// summed by one warp (lanes in G groups; group g holds the load components
// jj in [g * NJG, (g + 1) * NJG) of all NC point-load components and
// strides over the panel's nodes; each group's partials are reduced in a
// fixed butterfly order) into part[q][c * NJ + jj]; then, per pair, the
// panel sums added in grid order (k_pair_sum).  Neither order depends on
// how panels were grouped into waves.  The kernel is bound by the latency of
// its node loads, so each lane loads its next node before it computes the
// current one.
template <int P, int KC>
struct AccumShape {
  static constexpr int K = n_nodes(P);
  static constexpr int NJ = 3 * K;
  static constexpr int NC = KC == KD_HE ? 6 : 3;
  static constexpr int NOUT = NC * NJ;
  static constexpr int G = NOUT <= 27 ? 1 : (NOUT <= 54 ? 2 : 4);   // lane groups
  static constexpr int NJG = (NJ + G - 1) / G;
  static constexpr int LANES = 32 / G;
};

constexpr int ACCUM_WARPS = 4;

template <int P, int KC>
__global__ void __launch_bounds__(32 * ACCUM_WARPS, P == 0 ? ACCUM_MIN_BLOCKS : 1)
k_accum(int np, int64_t lo, const double* __restrict__ obs, const int* __restrict__ pair_oc,
        const int* __restrict__ pan_pair, const long long* __restrict__ pan_noff,
        const Hdr* __restrict__ hdr, const double* __restrict__ npx,
        const double* __restrict__ npy, const double* __restrict__ nw,
        const double* __restrict__ load, long long cap, const double* __restrict__ foot,
        double mu, double lam, double* __restrict__ part) {
  using A = AccumShape<P, KC>;
  constexpr int NJ = A::NJ, NC = A::NC, NJG = A::NJG, LANES = A::LANES, NOUT = A::NOUT;
  const Material m = make_material(mu, lam);
  const long long q0 = hdr->wave_q0, q1 = hdr->wave_q1, n0 = hdr->wave_n0;
  const int lane = threadIdx.x & 31;
  const int grp = lane / LANES, gl = lane % LANES;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q = q0 + warp; q < q1; q += nwarps) {
    const int i = pan_pair[q];
    const int64_t o = lo + pair_oc[i];
    const double xh0 = obs[3 * o], xh1 = obs[3 * o + 1];
    const double zeta = -obs[3 * o + 2] > 0.0 ? -obs[3 * o + 2] : 0.0;
    double sh[NJG];
#pragma unroll
    for (int t = 0; t < NJG; ++t) {
      const int jj = grp * NJG + t;
      sh[t] = jj < NJ ? foot[(size_t)i * NJ + jj] : 0.0;
    }
    double pt[NC][NJG];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int t = 0; t < NJG; ++t) pt[c][t] = 0.0;
    const long long ua = pan_noff[q] - n0, ub = pan_noff[q + 1] - n0;
    // the next node's data is loaded before this node's products, so each
    // lane keeps two nodes' loads in flight
    long long u = ua + gl;
    double px = 0.0, py = 0.0, w = 0.0, lv[NJG];
#pragma unroll
    for (int t = 0; t < NJG; ++t) lv[t] = 0.0;
    if (u < ub) {
      px = npx[u];
      py = npy[u];
      w = nw[u];
#pragma unroll
      for (int t = 0; t < NJG; ++t) {
        const int jj = grp * NJG + t;
        lv[t] = jj < NJ ? load[(size_t)jj * cap + u] : 0.0;
      }
    }
#pragma unroll 1
    for (; u < ub; u += LANES) {
      const long long un = u + LANES;
      double pxn = 0.0, pyn = 0.0, wn = 0.0, lvn[NJG];
#pragma unroll
      for (int t = 0; t < NJG; ++t) lvn[t] = 0.0;
      if (un < ub) {
        pxn = npx[un];
        pyn = npy[un];
        wn = nw[un];
#pragma unroll
        for (int t = 0; t < NJG; ++t) {
          const int jj = grp * NJG + t;
          lvn[t] = jj < NJ ? load[(size_t)jj * cap + un] : 0.0;
        }
      }
      double Bv[NC];
      if constexpr (KC == KD_HE) point_stress6_rcp(xh0 - px, xh1 - py, zeta, m.nu_f, Bv);
      else point_disp3_rcp(xh0 - px, xh1 - py, zeta, m.mu, m.nu_f, Bv);
#pragma unroll
      for (int c = 0; c < NC; ++c) Bv[c] *= w;
#pragma unroll
      for (int t = 0; t < NJG; ++t) {
        const int jj = grp * NJG + t;
        if (jj < NJ) {
          const double sv = lv[t] - sh[t];
#pragma unroll
          for (int c = 0; c < NC; ++c) pt[c][t] += Bv[c] * sv;
        }
      }
      px = pxn;
      py = pyn;
      w = wn;
#pragma unroll
      for (int t = 0; t < NJG; ++t) lv[t] = lvn[t];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int t = 0; t < NJG; ++t) {
        double v = pt[c][t];
#pragma unroll
        for (int d = LANES / 2; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        const int jj = grp * NJG + t;
        if (gl == 0 && jj < NJ) part[(size_t)q * NOUT + c * NJ + jj] = v;
      }
  }
}

// Per pair and output component: the pair's panel sums in grid order.
template <int P, int KC>
__global__ void __launch_bounds__(128)
k_pair_sum(int np, const long long* __restrict__ pair_poff, const double* __restrict__ part,
           double* __restrict__ acc) {
  constexpr int NOUT = AccumShape<P, KC>::NOUT;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)np * NOUT) return;
  const int i = (int)(t / NOUT), k = (int)(t % NOUT);
  double a = 0.0;
  for (long long q = pair_poff[i]; q < pair_poff[i + 1]; ++q) a += part[(size_t)q * NOUT + k];
  acc[(size_t)i * NOUT + k] = a;
}

// Per pair: the disk term of the grid's outer radius and the add into the
// pair's table row.
template <int P, int KC>
__global__ void __launch_bounds__(128)
k_finish(int np, int64_t lo, int64_t n_src, const double* __restrict__ obs,
         const SrcPrep* __restrict__ prep, const int* __restrict__ st_src,
         const int* __restrict__ pair_st, const int* __restrict__ pair_oc,
         const double* __restrict__ foot, const double* __restrict__ acc, double mu, double lam,
         double* __restrict__ T) {
  using A = AccumShape<P, KC>;
  constexpr int K = n_nodes(P), NJ = A::NJ;
  constexpr int NR = row_of(KC);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int s = st_src[pair_st[i]];
  const SrcPrep& sp = prep[s];
  const int oc = pair_oc[i];
  FoldPair fp;
  pair_geom(obs, lo, oc, sp, fp);
  double br[FOLD_MAX_BREAKS];
  double R1 = 0.0;
  if (fold_breaks(fp.rho_s, fp.zeta, sp.r_f, sp.eps, sp.diam, br, &R1) < 0) return;
  const Material m = make_material(mu, lam);
  const double* a = acc + (size_t)i * A::NOUT;
  const double* sh = foot + (size_t)i * NJ;
  double* row = T + (((int64_t)oc * n_src + s) * K) * NR;
  if constexpr (KC == KD_HE) {
    double srr, szz;
    disk_stress(R1, fp.zeta, m.nu_f, &srr, &szz);
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int k = 0; k < K; ++k)
      for (int mm = 0; mm < 3; ++mm) {
        double Hb[3][3];
        for (int c = 0; c < 6; ++c) {
          const double v = a[c * NJ + 3 * k + mm];
          Hb[ia[c]][ib[c]] = v;
          Hb[ib[c]][ia[c]] = v;
        }
        const double shv = sh[3 * k + mm];
        Hb[0][0] += shv * srr;
        Hb[1][1] += shv * srr;
        Hb[2][2] += shv * szz;
        for (int aa = 0; aa < 3; ++aa)
          for (int b = 0; b < 3; ++b) row[k * NR + 9 * aa + 3 * b + mm] += Hb[aa][b];
      }
  } else {
    const double uz = disk_disp_z(R1, fp.zeta, m.mu, m.nu_f);
    for (int k = 0; k < K; ++k)
      for (int mm = 0; mm < 3; ++mm)
        for (int ii = 0; ii < 3; ++ii)
          row[k * NR + 3 * ii + mm] += a[ii * NJ + 3 * k + mm] +
                                       (ii == 2 ? sh[3 * k + mm] * uz : 0.0);
  }
}

__global__ void k_zero(double* __restrict__ a, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = 0.0;
}

__global__ void k_census_pairs(const Hdr* __restrict__ hdr, unsigned long long* __restrict__ census,
                               int np) {
  census[MHS_CENSUS_PAIRS] += (unsigned long long)np;
  census[MHS_CENSUS_PANELS] += (unsigned long long)hdr->q_batch;
}

}  // namespace fold_waves

namespace fold_waves {

// Bytes of the fold region's parts.
template <int P, int KC, class RF>
struct Sizes {
  static constexpr int K = n_nodes(P), NJ = 3 * K;
  static constexpr int NOUT = AccumShape<P, KC>::NOUT;
  static constexpr size_t per_src = sizeof(Src<P, RF>);
  // pair_st, pair_oc (int), pair_poff, pair_noff (scan input and output,
  // one more entry), foot (NJ), acc (NOUT)
  static constexpr size_t per_pair = 4 + 4 + 8 + 8 + 8 * NJ + 8 * NOUT;
  static constexpr size_t per_panel = 8 + 8 + 8 + 4 + 8 * NOUT;   // ra, rb, first node, pair, sums
  static constexpr size_t per_node = 8 * 3 + 4 + 1 + 4 + 8 * NJ;
};

inline size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// The fold of one observer chunk: plan, then batches of band pairs, each
// in waves of whole panels.  Returns an MHS status code.
template <int P, int KC, class RF>
int run_fold(const mhs_request* r, cudaStream_t st, char* region, size_t region_bytes,
             int64_t lo, int64_t nc, const SrcPrep* prep, const int* cnt, const int* list,
             double* T, int* status, unsigned long long* census, const Tune& tune) {
  using Z = Sizes<P, KC, RF>;
  constexpr int NJ = Z::NJ;
  constexpr int NOUT = Z::NOUT;
  const int64_t n_src = r->n_src;
  int dev = 0, sms = 0;
  MHS_CUDA_TRY(cudaGetDevice(&dev));
  MHS_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // fixed part: header and the straddler tables
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    char* p = region + off;
    off = up256(off + bytes);
    return p;
  };
  Hdr* hdr = (Hdr*)carve(sizeof(Hdr));
  int* st_rank = (int*)carve(sizeof(int) * n_src);
  int* st_src = (int*)carve(sizeof(int) * n_src);
  long long* st_off = (long long*)carve(sizeof(long long) * (n_src + 1));
  if (off >= region_bytes)
    return fail(MHS_ERR_WORKSPACE, "fold region of %zu bytes below its fixed part", region_bytes);
  MHS_CUDA_TRY(cudaMemsetAsync(hdr, 0, sizeof(Hdr), st));
  {
    StageTimer t(MHS_STAGE_FOLD_PLAN, st);
    k_band_scan<<<1, 1024, 0, st>>>(n_src, prep, cnt, st_rank, st_src, st_off, hdr);
    count_kernels(1);
  }
  Hdr h;
  MHS_CUDA_TRY(cudaMemcpyAsync(&h, hdr, sizeof(Hdr), cudaMemcpyDeviceToHost, st));
  MHS_CUDA_TRY(cudaStreamSynchronize(st));
  if (h.n_pairs == 0) return MHS_OK;
  std::vector<long long> so((size_t)h.n_st + 1);
  MHS_CUDA_TRY(cudaMemcpyAsync(so.data(), st_off, sizeof(long long) * so.size(),
                               cudaMemcpyDeviceToHost, st));
  MHS_CUDA_TRY(cudaStreamSynchronize(st));
  // budgets of the variable part
  const size_t rest = region_bytes - off;
  const size_t b_src = rest / 10, b_pair = rest * 3 / 20, b_pan = rest * 3 / 20;
  const size_t b_node = rest - b_src - b_pair - b_pan - 24 * 256;   // 19 aligned carves below
  const long long cap_src = (long long)(b_src / Z::per_src);
  const long long cap_pair = (long long)(b_pair / Z::per_pair) - 2;
  const long long cap_pan = (long long)(b_pan / Z::per_panel) - 2;
  const long long cap_node = (long long)(b_node / Z::per_node);
  if (cap_src < 1 || cap_pair < 1 || cap_pan < 1 || cap_node < 1)
    return fail(MHS_ERR_WORKSPACE, "fold region of %zu bytes too small for one pair", region_bytes);
  Src<P, RF>* srcs = (Src<P, RF>*)carve(Z::per_src * cap_src);
  int* pair_st = (int*)carve(4 * cap_pair);
  int* pair_oc = (int*)carve(4 * cap_pair);
  long long* pair_poff = (long long*)carve(8 * (cap_pair + 1));
  long long* pair_noff = (long long*)carve(8 * (cap_pair + 1));
  double* foot = (double*)carve(8 * NJ * cap_pair);
  double* acc = (double*)carve(8 * NOUT * cap_pair);
  double* pan_ra = (double*)carve(8 * cap_pan);
  double* pan_rb = (double*)carve(8 * cap_pan);
  long long* pan_noff = (long long*)carve(8 * (cap_pan + 1));
  int* pan_pair = (int*)carve(4 * cap_pan);
  double* pan_sum = (double*)carve(8 * NOUT * cap_pan);
  double* npx = (double*)carve(8 * cap_node);
  double* npy = (double*)carve(8 * cap_node);
  double* nw = (double*)carve(8 * cap_node);
  int* npair = (int*)carve(4 * cap_node);
  unsigned char* ncls = (unsigned char*)carve(cap_node);
  int* nlist = (int*)carve(4 * cap_node);
  double* load = (double*)carve(8 * NJ * cap_node);
  if (off > region_bytes) return fail(MHS_ERR_WORKSPACE, "fold region carve-up overflow");
  const SurfaceLoadConsts* slcs = &srcs[0].slc;
  // grid sizes of the grid-stride kernels
  int occ_far = 1, occ_near = 1, occ_nodes = 1;
  MHS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_far, k_far<P, KC, RF>, 128, 0));
  MHS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_near, k_near<P, KC>, 128, 0));
  MHS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_nodes, k_nodes<P>, 256, 0));
  const int g_far = sms * (occ_far > 0 ? occ_far : 1) * tune.far_mult;
  const int g_near = sms * (occ_near > 0 ? occ_near : 1) * tune.near_mult;
  const int g_nodes = sms * (occ_nodes > 0 ? occ_nodes : 1) * 2;
  const int g_scatter = sms * 8;
  // closed-form near field out to D_STAR element lengths in both forms (a
  // near node's FP64 closed form costs less than the float 12 x 12 rule)
  const double near_l = cst::D_STAR;
  long long p0 = 0;
  long long batch = cap_pair;
  while (p0 < h.n_pairs) {
    long long p1 = std::min<long long>(h.n_pairs, p0 + batch);
    // straddlers the batch touches, within the source-data capacity
    auto strad = [&](long long p) {  // straddle rank of pair p
      return (long long)(std::upper_bound(so.begin(), so.end(), p) - so.begin()) - 1;
    };
    const long long j0 = strad(p0);
    if (strad(p1 - 1) - j0 + 1 > cap_src) p1 = std::max<long long>(p0 + 1, so[j0 + cap_src]);
    const int np = (int)(p1 - p0);
    const long long j1 = strad(p1 - 1) + 1;
    MHS_CUDA_TRY(cudaMemsetAsync(&hdr->max_panel, 0, sizeof(long long), st));
    {
      StageTimer t(MHS_STAGE_FOLD_PLAN, st);
      k_pairs<<<(np + 127) / 128, 128, 0, st>>>(p0, np, lo, nc, r->obs, prep, list, st_src, st_off,
                                                hdr, pair_st, pair_oc, pair_poff, pair_noff, status);
      k_scan<<<1, 1024, 0, st>>>(pair_poff, np, &hdr->q_batch, nullptr);
      k_scan<<<1, 1024, 0, st>>>(pair_noff, np, &hdr->n_batch, nullptr);
      count_kernels(3);
    }
    MHS_CUDA_TRY(cudaMemcpyAsync(&h, hdr, sizeof(Hdr), cudaMemcpyDeviceToHost, st));
    MHS_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.q_batch > cap_pan) {
      if (np == 1)
        return fail(MHS_ERR_WORKSPACE, "one fold pair has %lld panels, above the fold region's "
                    "%lld", h.q_batch, cap_pan);
      batch = std::max<long long>(1, np / 2);
      continue;
    }
    if (h.max_panel > cap_node / 2)
      return fail(MHS_ERR_WORKSPACE, "a fold panel of %lld nodes does not fit the fold "
                  "region's %lld-node waves", h.max_panel, cap_node);
    const long long nq = h.q_batch, nn = h.n_batch;
    {
      StageTimer t(MHS_STAGE_FOLD_PLAN, st);
      k_src<P, KC, RF><<<(unsigned)(j1 - j0), 128, 0, st>>>((int)j0, (int)(j1 - j0), st_src, prep,
                                                            r->mu, r->lam, srcs);
      k_panels<<<(np + 1 + 127) / 128, 128, 0, st>>>(np, lo, r->obs, prep, st_src, pair_st,
                                                     pair_oc, pair_poff, pair_noff, pan_ra, pan_rb,
                                                     pan_noff, pan_pair);
      k_foot<P, KC, RF><<<(np + 127) / 128, 128, 0, st>>>(np, (int)j0, lo, r->obs, prep, st_src,
                                                          pair_st, pair_oc, srcs, foot);
      count_kernels(3);
      if (census) {
        k_census_pairs<<<1, 1, 0, st>>>(hdr, census, np);
        count_kernels(1);
      }
    }
    const long long span = cap_node - h.max_panel;
    const long long waves = (nn + span - 1) / span;
    for (long long w = 0; w < waves; ++w) {
      {
        StageTimer t(MHS_STAGE_FOLD_NODES, st);
        k_wave_begin<<<1, 1, 0, st>>>(w, span, nq, pan_noff, hdr);
        k_nodes<P><<<g_nodes, 256, 0, st>>>(near_l, np, lo, r->obs, prep, st_src, pair_st,
                                            pair_oc, pan_pair, pan_ra, pan_rb, pan_noff, hdr, npx,
                                            npy, nw, npair, ncls);
        k_count<<<g_scatter, 256, 0, st>>>(hdr, ncls);
        k_wave_classes<<<1, 1, 0, st>>>(hdr, census);
        k_scatter<<<g_scatter, 256, 0, st>>>(hdr, ncls, nlist);
        count_kernels(5);
      }
      {
        StageTimer t(MHS_STAGE_FOLD_FAR, st);
        k_far<P, KC, RF><<<g_far, 128, 0, st>>>(hdr, nlist, npx, npy, npair, pair_st, (int)j0,
                                                st_src, prep, srcs, load, cap_node);
        count_kernels(1);
      }
      {
        StageTimer t(MHS_STAGE_FOLD_NEAR, st);
        k_near<P, KC><<<g_near, 128, 0, st>>>(hdr, nlist, npx, npy, npair, pair_st, (int)j0,
                                              st_src, prep, slcs, (long long)sizeof(Src<P, RF>),
                                              load, cap_node);
        count_kernels(1);
      }
      {
        StageTimer t(MHS_STAGE_FOLD_ACCUM, st);
        k_accum<P, KC><<<sms * 16, 32 * ACCUM_WARPS, 0, st>>>(np, lo, r->obs, pair_oc, pan_pair,
                                                             pan_noff, hdr, npx, npy, nw, load,
                                                             cap_node, foot, r->mu, r->lam,
                                                             pan_sum);
        count_kernels(1);
      }
    }
    {
      StageTimer t(MHS_STAGE_FOLD_ACCUM, st);
      const long long nt = (long long)np * NOUT;
      k_pair_sum<P, KC><<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(np, pair_poff, pan_sum, acc);
      count_kernels(1);
      k_finish<P, KC><<<(np + 127) / 128, 128, 0, st>>>(np, lo, n_src, r->obs, prep, st_src,
                                                        pair_st, pair_oc, foot, acc, r->mu, r->lam,
                                                        T);
      count_kernels(1);
    }
    MHS_CUDA_TRY(cudaGetLastError());
    p0 = p1;
    batch = cap_pair;
  }
  return MHS_OK;
}

}  // namespace fold_waves
