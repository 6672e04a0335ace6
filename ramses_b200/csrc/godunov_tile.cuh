// godunov_tile.cuh -- the level-wide godunov kernel (godunov_fine.f90:5-35,
// godfine1 :486-911 and unsplit, umuscl.f90:22-171) as a tiled sm_100a stencil.
//
// A tile is an aligned box of TX x TY x TZ level-l cells (TX/2 x TY/2 x TZ/2
// octs). One CTA owns one tile:
//   A. gather the (TX+4)(TY+4)(TZ+4) stencil into shared memory as primitive
//      variables. Each 2x2x2 block of the stencil is an existing level-l oct
//      (read from uold), a prolongated coarse cell (interpol_hydro, computed
//      beforehand into the interpolation buffer), or absent (no active oct
//      reads it); plus the refinement flag son(cell)>0 of every cell;
//   B. slopes + MUSCL-Hancock trace once per cell of the tile and of the
//      one-cell face slabs around it;
//   C. one Riemann problem per face, flux*dt/dx, zeroed where either side is
//      refined (godunov_fine.f90:720-747);
//   D. unew += (Fx_l - Fx_r) then y then z for the cells of active octs
//      (godunov_fine.f90:751-792);
//   E. the boundary-face fluxes of octs that border an unrefined coarser cell
//      are stored for the deterministic fine-to-coarse correction.
// Every quantity is a pure function of its stencil, so computing each cell
// and face once per tile gives the values the reference computes (redundantly)
// per oct.
#pragma once
#include <cstdint>

#include "cp_async.cuh"
#include "hydro_core.cuh"

namespace rb {

struct TileArgs {
  const double* __restrict__ uold;      // [5][ncell], device cell layout
  double* __restrict__ unew;            // [5][ncell]
  const int32_t* __restrict__ son;      // [ncell], device cell layout
  const double* __restrict__ interp;    // [5][ninterp*8] prolongated blocks
  const int32_t* __restrict__ tile_blk; // [ntile][NBLK] block codes
  const int32_t* __restrict__ tile_corr_off; // [ntile+1] (null: no correction slots)
  const int32_t* __restrict__ tile_corr;     // [entries][2] (oct in tile | face << 8, slot): the
                                             // faces whose fluxes the fine-to-coarse correction reads
  double* __restrict__ corr_flux;       // [nslot][6][4][5]
  int64_t ncell;
  int64_t ninterp8;                     // ninterp*8 (stride of interp)
  int32_t ncoarse;
  int32_t ntile;
  int32_t has_refined;                  // any son>0 among this level's cells
  int32_t dx_pow2;                      // dx is an exact power of two
  int32_t fused;                        // 1: unew = uold + fluxes (set_unew fused) and
                                        //    CFL partials of the new state; 2: unew = uold +
                                        //    fluxes only (a level without finer octs, whose
                                        //    unew holds no fine-to-coarse correction)
  double dt, dx, inv_dx;
  const double* __restrict__ dt_dev;    // if non-null, dt is read here
  double* __restrict__ partial;         // fused: [ntile][4] (min dt, mass, E, eint)
  const double* __restrict__ gate;      // if non-null and *gate != 0 the launch is a no-op
  double* __restrict__ divu;            // pressure_fix (PF kernels): [ncell] velocity divergence
  double* __restrict__ enew;            //   and internal energy, updated like unew
  double* __restrict__ corr_tmp;        //   [nslot][6][4][2] their correction-face fluxes
  rb_hydro_params hp;
};

// block code: >= 0 oct index (igrid-1); -1 absent; <= -2 interpolation entry (-code-2)
template <int TX, int TY, int TZ>
struct TileGeom {
  static constexpr int SX = TX + 4, SY = TY + 4, SZ = TZ + 4;
  static constexpr int NS = SX * SY * SZ;
  static constexpr int BX = TX / 2 + 2, BY = TY / 2 + 2, BZ = TZ / 2 + 2;
  static constexpr int NBLK = BX * BY * BZ;
  // face-state arrays (per variable)
  static constexpr int NFX = (TX + 1) * TY * TZ;
  static constexpr int NFY = TX * (TY + 1) * TZ;
  static constexpr int NFZ = TX * TY * (TZ + 1);
  static constexpr int NF = NFX + NFY + NFZ;
  static constexpr int NCELL = TX * TY * TZ;
  static constexpr int NTRACE = NCELL + 2 * (TY * TZ + TX * TZ + TX * TY);
  static_assert(5 * NF <= 5 * NS, "flux must fit in the stencil buffer");
};

// Stencil cells read by the slopes of types 0, 1, 2, 7 and 8: the tile, its
// one-cell face slabs and their six neighbours. Listed block-major as
// (block << 3 | child): all children of a block with at most one halo
// coordinate, the two inner-layer children of an edge block (two halo
// coordinates), nothing of a corner block.
template <int TX, int TY, int TZ>
constexpr int gather_children(int b, int ch) {
  using G = TileGeom<TX, TY, TZ>;
  const int bx = b % G::BX, by = (b / G::BX) % G::BY, bz = b / (G::BX * G::BY);
  const bool hx = bx == 0 || bx == G::BX - 1, hy = by == 0 || by == G::BY - 1, hz = bz == 0 || bz == G::BZ - 1;
  const int nh = (int)hx + (int)hy + (int)hz;
  if (nh <= 1) return 1;
  if (nh == 3) return 0;
  // inner layer: child 1 of the first block, child 0 of the last
  const int px = ch & 1, py = (ch >> 1) & 1, pz = ch >> 2;
  if (hx && px != (bx == 0 ? 1 : 0)) return 0;
  if (hy && py != (by == 0 ? 1 : 0)) return 0;
  if (hz && pz != (bz == 0 ? 1 : 0)) return 0;
  return 1;
}
template <int TX, int TY, int TZ>
constexpr int gather_count() {
  int n = 0;
  for (int b = 0; b < TileGeom<TX, TY, TZ>::NBLK; b++)
    for (int ch = 0; ch < 8; ch++) n += gather_children<TX, TY, TZ>(b, ch);
  return n;
}
template <int TX, int TY, int TZ>
struct GatherList {
  static constexpr int N = gather_count<TX, TY, TZ>();
  uint16_t e[N];
  constexpr GatherList() : e{} {
    int n = 0;
    for (int b = 0; b < TileGeom<TX, TY, TZ>::NBLK; b++)
      for (int ch = 0; ch < 8; ch++)
        if (gather_children<TX, TY, TZ>(b, ch)) e[n++] = (uint16_t)(b << 3 | ch);
  }
};
template <int TX, int TY, int TZ>
__device__ const GatherList<TX, TY, TZ> kGatherList{};

template <typename R, int TX, int TY, int TZ>
constexpr size_t tile_smem_bytes() {
  using G = TileGeom<TX, TY, TZ>;
  // q/flux union + face states (M and P) + block codes + refinement flags
  return sizeof(R) * (size_t)(5 * G::NS) + sizeof(R) * (size_t)(2 * 5 * G::NF) +
         sizeof(int32_t) * (size_t)G::NBLK + (size_t)((G::NS + 15) & ~15);
}

// RS (Riemann solver) and ST (slope type) fix the scheme at compile time;
// RS = 0 / ST = -1 read it from a.hp at run time. PF: pressure_fix, the
// velocity-divergence and internal-energy fluxes of every face (umuscl.f90
// cmpflxm's tmp, :845-849) update a.divu and a.enew beside unew
// (godunov_fine.f90:735-744, 775-789).
template <typename R, int TX, int TY, int TZ, int NT, int RS, int ST, bool PF = false>
__global__ void __launch_bounds__(NT) godunov_tile_kernel(TileArgs a) {
  using G = TileGeom<TX, TY, TZ>;
  constexpr int SX = G::SX, SY = G::SY, NS = G::NS;
  constexpr int BX = G::BX, BY = G::BY, NBLK = G::NBLK;
  constexpr int NFX = G::NFX, NFY = G::NFY, NF = G::NF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* q = reinterpret_cast<R*>(smem_raw);                 // [5][NS]; reused as flux [5][NF]
  R* qm = q + 5 * NS;                                    // [5][NF]
  R* qp = qm + 5 * NF;                                   // [5][NF]
  int32_t* blk = reinterpret_cast<int32_t*>(qp + 5 * NF);// [NBLK]
  unsigned char* okf = reinterpret_cast<unsigned char*>(blk + NBLK);  // [NS]

  const int tile = blockIdx.x;
  if (tile >= a.ntile) return;
  const int tid = threadIdx.x;
  const Consts<R> c = make_consts<R>(a.hp);
  const int64_t ncell = a.ncell;

  constexpr int NOCT = (TX / 2) * (TY / 2) * (TZ / 2);
  __shared__ int32_t corr_range[2];
  __shared__ int32_t corr_ent[2 * 6 * NOCT];
  // the gate (the device scheduler's end-of-run flag) is read together with
  // the tile's codes, so that the two loads overlap; every thread reads the
  // same value, so the return is uniform and precedes the barrier
  const double gate = a.gate != nullptr ? *a.gate : 0.0;
  for (int i = tid; i < NBLK; i += NT) blk[i] = a.tile_blk[(int64_t)tile * NBLK + i];
  if (a.tile_corr_off != nullptr && tid < 2) corr_range[tid] = a.tile_corr_off[tile + tid];
  if (gate != 0.0) return;
  __syncthreads();

  // the tile's correction-face entries are copied to shared memory while the
  // tile is computed (they are read at the end)
  if (a.tile_corr_off != nullptr)
    for (int i = tid; i < 2 * (corr_range[1] - corr_range[0]); i += NT)
      cp_async4(corr_ent + i, a.tile_corr + 2 * corr_range[0] + i);
  cp_async_commit();

  // ---- A. gather + ctoprim ------------------------------------------------
  const int slope_type = ST >= 0 ? ST % 10 : a.hp.slope_type;
  const bool slope27 = (slope_type == 3);
  // the 27-point slopes and the corner divergence of difmag read the edge and
  // corner cells of the stencil too
  const bool full_gather = slope27 || (RS == 0 && a.hp.difmag > 0.0);
  // one stencil cell: its raw state is loaded by gather_cell and converted by
  // put_cell (the listed gather keeps the loads of two cells in flight
  // before their conversion). Blocks coded -1 are read by no present cell:
  // only their flags are set.
  auto gather_cell = [&](int b, int ch, double u[5], int& code, int& sonv, int& inner) -> int {
    const int bx = b % BX, by = (b / BX) % BY, bz = b / (BX * BY);
    const int sx = 2 * bx + (ch & 1), sy = 2 * by + ((ch >> 1) & 1), sz = 2 * bz + (ch >> 2);
    code = blk[b];
    sonv = 0;
    // L2-only loads: the tile reads each stencil cell once, and leaving L1
    // to the loads in flight lets more of them be outstanding
    if (code >= 0) {
      const int64_t dc = (int64_t)a.ncoarse + (int64_t)code * 8 + ch;
#pragma unroll
      for (int v = 0; v < 5; v++) u[v] = __ldcg(a.uold + v * ncell + dc);
      if (a.has_refined) sonv = __ldcg(a.son + dc);
    } else if (code <= -2) {
      const int64_t e = (int64_t)(-code - 2) * 8 + ch;
#pragma unroll
      for (int v = 0; v < 5; v++) u[v] = __ldcg(a.interp + v * a.ninterp8 + e);
    }
    // a tile-interior cell of a present oct (its faces and update are used)
    inner = sx >= 2 && sx < 2 + TX && sy >= 2 && sy < 2 + TY && sz >= 2 && sz < 2 + TZ && code >= 0;
    return sx + SX * (sy + SY * sz);
  };
  auto put_cell = [&](int s, const double u[5], int code, int sonv, int inner) {
    // okf bit 0: the cell is refined (its faces carry no flux); bit 1: a
    // tile-interior cell of a present oct
    okf[s] = (unsigned char)((sonv > 0 ? 1 : 0) | (inner ? 2 : 0));
    if (code == -1) return;
    const Prim<R> pq = ctoprim_cell<R>(u, a.hp);
    q[0 * NS + s] = pq.r;
    q[1 * NS + s] = pq.u;
    q[2 * NS + s] = pq.v;
    q[3 * NS + s] = pq.w;
    q[4 * NS + s] = pq.p;
  };
  if (!full_gather) {
    using GL = GatherList<TX, TY, TZ>;
    constexpr int NG = GL::N;
    constexpr int PER = (NG + NT - 1) / NT;
    constexpr int NB = PER < 2 ? PER : 2;
    for (int j0 = 0; j0 < PER; j0 += NB) {
      double u[NB][5];
      int sidx[NB], code[NB], sonv[NB], inner[NB];
#pragma unroll
      for (int j = 0; j < NB; j++) {
        const int it = tid + (j0 + j) * NT;
        sidx[j] = -1;
        if (j0 + j < PER && it < NG) {
          const int e = __ldg(&kGatherList<TX, TY, TZ>.e[it]);
          sidx[j] = gather_cell(e >> 3, e & 7, u[j], code[j], sonv[j], inner[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < NB; j++)
        if (sidx[j] >= 0) put_cell(sidx[j], u[j], code[j], sonv[j], inner[j]);
    }
  } else {
    // every cell of the stencil
    for (int it = tid; it < NBLK * 8; it += NT) {
      double u[5];
      int code, sonv, inner;
      const int s = gather_cell(it >> 3, it & 7, u, code, sonv, inner);
      put_cell(s, u, code, sonv, inner);
    }
  }
  __syncthreads();

  // ---- B. slopes + trace ----------------------------------------------------
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;
  R dtd[3];
  {
    const double dtdx = dt / a.dx;  // trace3d.f90 dtdx = dt/dx (dx=dy=dz)
    dtd[0] = dtd[1] = dtd[2] = (R)dtdx;
  }
  // present(x,y,z): the tile-interior cell belongs to an oct of this level
  // (its update and its faces are used; bit 1 of okf). A block coded -1 is
  // absent and not a stencil source of any present oct, so no face touching
  // it is used.
  auto present = [&](int x, int y, int z) { return (okf[(x + 2) + SX * ((y + 2) + SY * (z + 2))] & 2) != 0; };
  for (int it = tid; it < G::NTRACE; it += NT) {
    int x, y, z;
    unsigned mask;
    if (it < G::NCELL) {
      x = it % TX; y = (it / TX) % TY; z = it / (TX * TY); mask = 7u;
      if (blk[(x / 2 + 1) + BX * ((y / 2 + 1) + BY * (z / 2 + 1))] == -1) continue;
    } else {
      int r = it - G::NCELL;
      if (r < 2 * TY * TZ) {           // x slabs: x = -1 (qm only) and x = TX (qp only)
        const int side = r / (TY * TZ); r %= TY * TZ;
        x = side ? TX : -1; y = r % TY; z = r / TY; mask = 1u;
        if (!present(side ? TX - 1 : 0, y, z)) continue;
      } else if ((r -= 2 * TY * TZ) < 2 * TX * TZ) {
        const int side = r / (TX * TZ); r %= TX * TZ;
        y = side ? TY : -1; x = r % TX; z = r / TX; mask = 2u;
        if (!present(x, side ? TY - 1 : 0, z)) continue;
      } else {
        r -= 2 * TX * TZ;
        const int side = r / (TX * TY); r %= TX * TY;
        z = side ? TZ : -1; x = r % TX; y = r / TX; mask = 4u;
        if (!present(x, y, side ? TZ - 1 : 0)) continue;
      }
    }
    const int s = (x + 2) + SX * ((y + 2) + SY * (z + 2));
    R dq[5][3];
    Prim<R> q0;
    q0.r = q[s]; q0.u = q[NS + s]; q0.v = q[2 * NS + s]; q0.w = q[3 * NS + s]; q0.p = q[4 * NS + s];
    if (slope_type == 0) {
#pragma unroll
      for (int v = 0; v < 5; v++) { dq[v][0] = (R)0; dq[v][1] = (R)0; dq[v][2] = (R)0; }
    } else if (!slope27) {
      constexpr int st[3] = {1, SX, SX * SY};
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const R* qv = q + v * NS;
        const R qc = qv[s];
#pragma unroll
        for (int d = 0; d < 3; d++)
          dq[v][d] = slope1<R>(qv[s - st[d]], qc, qv[s + st[d]], slope_type, c.slope_theta);
      }
    } else {
      // positivity-preserving multidimensional slope (umuscl.f90:1328-1392)
      const R half = (R)0.5, one = (R)1, zero = (R)0;
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const R* qv = q + v * NS;
        const R qc = qv[s];
        R vmin = (R)0, vmax = (R)0;
        bool first = true;
        for (int kk = -1; kk <= 1; kk++)
          for (int ii = -1; ii <= 1; ii++)
            for (int jj = -1; jj <= 1; jj++) {
              const R d = qv[s + ii + SX * (jj + SY * kk)] - qc;
              if (first) { vmin = d; vmax = d; first = false; }
              else { vmin = fmn(vmin, d); vmax = fmx(vmax, d); }
            }
        const R dfx = half * (qv[s + 1] - qv[s - 1]);
        const R dfy = half * (qv[s + SX] - qv[s - SX]);
        const R dfz = half * (qv[s + SX * SY] - qv[s - SX * SY]);
        const R dff = half * ((R)fabs(dfx) + (R)fabs(dfy) + (R)fabs(dfz));
        R slop;
        if (dff > zero) slop = fmn(one, fmn((R)fabs(vmin), (R)fabs(vmax)) / dff);
        else slop = one;
        dq[v][0] = slop * dfx; dq[v][1] = slop * dfy; dq[v][2] = slop * dfz;
      }
    }
    Prim<R> sp[3], sm[3];
    trace_sel<R, RS, ST>(q0, dq, c, dtd, sp, sm, mask);
    // store: qm of direction d at face index (coord+1), qp at face index coord
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (!(mask & (1u << d))) continue;
      int off, fm, fp;
      if (d == 0) { off = 0;         fm = (x + 1) + (TX + 1) * (y + TY * z); fp = x + (TX + 1) * (y + TY * z); }
      else if (d == 1) { off = NFX;  fm = x + TX * ((y + 1) + (TY + 1) * z); fp = x + TX * (y + (TY + 1) * z); }
      else { off = NFX + NFY;        fm = x + TX * (y + TY * (z + 1));       fp = x + TX * (y + TY * z); }
      const bool wm = (d == 0) ? (x < TX) : (d == 1) ? (y < TY) : (z < TZ);
      const bool wp = (d == 0) ? (x >= 0) : (d == 1) ? (y >= 0) : (z >= 0);
      if (wm) {
        qm[0 * NF + off + fm] = sm[d].r; qm[1 * NF + off + fm] = sm[d].u; qm[2 * NF + off + fm] = sm[d].v;
        qm[3 * NF + off + fm] = sm[d].w; qm[4 * NF + off + fm] = sm[d].p;
      }
      if (wp) {
        qp[0 * NF + off + fp] = sp[d].r; qp[1 * NF + off + fp] = sp[d].u; qp[2 * NF + off + fp] = sp[d].v;
        qp[3 * NF + off + fp] = sp[d].w; qp[4 * NF + off + fp] = sp[d].p;
      }
    }
  }
  // difmag > 0 (run-time scheme variant): cmpdivu (uplmde.f90:702-764), the
  // velocity divergence at the cell corners (x-1/2, y-1/2, z-1/2) of the tile,
  // x in 0..TX etc., from the primitive velocities, before phase C reuses q
  constexpr int CXN = TX + 1, CYN = TY + 1, NCORN = (TX + 1) * (TY + 1) * (TZ + 1);
  R* cdiv = nullptr;
  if constexpr (RS == 0) {
    __shared__ R cdiv_s[NCORN];
    cdiv = cdiv_s;
    if (a.hp.difmag > 0.0) {
      const R quarter = (R)0.5 * (R)0.5;
      const R fxd = (R)(quarter / (R)a.dx), fyd = fxd, fzd = fxd;
      for (int it = tid; it < NCORN; it += NT) {
        const int x = it % CXN, y = (it / CXN) % CYN, z = it / (CXN * CYN);
        auto Q = [&](int ox, int oy, int oz, int v) {
          return q[v * NS + (x + ox + 2) + SX * ((y + oy + 2) + SY * (z + oz + 2))];
        };
        R ux = (R)0, vy = (R)0, wz = (R)0;
        ux = ux + fxd * (Q(0, 0, 0, 1) - Q(-1, 0, 0, 1));
        ux = ux + fxd * (Q(0, -1, 0, 1) - Q(-1, -1, 0, 1));
        vy = vy + fyd * (Q(0, 0, 0, 2) - Q(0, -1, 0, 2) + Q(-1, 0, 0, 2) - Q(-1, -1, 0, 2));
        ux = ux + fxd * (Q(0, 0, -1, 1) - Q(-1, 0, -1, 1) + Q(0, -1, -1, 1) - Q(-1, -1, -1, 1));
        vy = vy + fyd * (Q(0, 0, -1, 2) - Q(0, -1, -1, 2) + Q(-1, 0, -1, 2) - Q(-1, -1, -1, 2));
        wz = wz + fzd * (Q(0, 0, 0, 3) - Q(0, 0, -1, 3) + Q(0, -1, 0, 3) - Q(0, -1, -1, 3) + Q(-1, 0, 0, 3) -
                         Q(-1, 0, -1, 3) + Q(-1, -1, 0, 3) - Q(-1, -1, -1, 3));
        cdiv[it] = ux + vy + wz;
      }
    }
  }
  __syncthreads();

  // ---- C. Riemann fluxes (flux buffer aliases q) ------------------------------
  // raw (conservative) state of stencil cell s, as phase A gathered it
  auto raw_cell = [&](int s, double u[5]) {
    const int sx = s % SX, sy = (s / SX) % SY, sz = s / (SX * SY);
    const int b = (sx >> 1) + BX * ((sy >> 1) + BY * (sz >> 1));
    const int ch = (sx & 1) + 2 * (sy & 1) + 4 * (sz & 1);
    const int code = blk[b];
    if (code >= 0) {
      const int64_t dc = (int64_t)a.ncoarse + (int64_t)code * 8 + ch;
      for (int v = 0; v < 5; v++) u[v] = __ldcg(a.uold + v * ncell + dc);
    } else if (code <= -2) {
      const int64_t e = (int64_t)(-code - 2) * 8 + ch;
      for (int v = 0; v < 5; v++) u[v] = __ldcg(a.interp + v * a.ninterp8 + e);
    } else {
      for (int v = 0; v < 5; v++) u[v] = 0.0;
    }
  };
  R* F = q;
  for (int f = tid; f < NF; f += NT) {
    int d, x, y, z;
    if (f < NFX) { d = 0; x = f % (TX + 1); y = (f / (TX + 1)) % TY; z = f / ((TX + 1) * TY); }
    else if (f < NFX + NFY) { const int r = f - NFX; d = 1; x = r % TX; y = (r / TX) % (TY + 1); z = r / (TX * (TY + 1)); }
    else { const int r = f - NFX - NFY; d = 2; x = r % TX; y = (r / TX) % TY; z = r / (TX * TY); }
    // the face between cell (x,y,z) and its lower neighbour along d is used
    // only when one of the two is a present cell
    const int sr = (x + 2) + SX * ((y + 2) + SY * (z + 2));
    const int sl = sr - (d == 0 ? 1 : d == 1 ? SX : SX * SY);
    const int fl = okf[sl] | okf[sr];
    if (!(fl & 2)) continue;
    Prim<R> L, Rr;
    L.r = qm[f]; L.u = qm[NF + f]; L.v = qm[2 * NF + f]; L.w = qm[3 * NF + f]; L.p = qm[4 * NF + f];
    Rr.r = qp[f]; Rr.u = qp[NF + f]; Rr.v = qp[2 * NF + f]; Rr.w = qp[3 * NF + f]; Rr.p = qp[4 * NF + f];
    R ql[5], qr[5], fg[6], fo[5];
    to_face(L, d, ql);
    to_face(Rr, d, qr);
    riemann_sel<R, RS>(ql, qr, c, fg);
    from_face(fg, d, fo);
    // refined interface: either neighbour cell refined -> zero flux
    const bool zero_face = (fl & 1) != 0;
    auto scaled = [&](R x) -> R {
      if (sizeof(R) == 8) {
        // flux = fx*dt/dx, evaluated as (fx*dt)/dx (umuscl.f90:101-163);
        // division by an exact power of two equals the multiplication
        const double t = (double)x * dt;
        return (R)(a.dx_pow2 ? t * a.inv_dx : t / a.dx);
      }
      return x * dtd[0];
    };
    if (RS == 0 && a.hp.difmag > 0.0) {
      // consup (uplmde.f90:769-866): + dt*difmag*min(0, div1)*(u_R - u_L)
      // with div1 the mean of the face's four corner divergences, added
      // before the refined-face zeroing
      const R quarter = (R)0.5 * (R)0.5;
      auto D = [&](int cx, int cy, int cz) { return cdiv[cx + CXN * (cy + CYN * cz)]; };
      R div1;
      if (d == 0) {
        div1 = quarter * D(x, y, z);
        div1 = div1 + quarter * D(x, y + 1, z);
        div1 = div1 + quarter * (D(x, y, z + 1) + D(x, y + 1, z + 1));
      } else if (d == 1) {
        div1 = (R)0;
        div1 = div1 + quarter * (D(x, y, z) + D(x + 1, y, z));
        div1 = div1 + quarter * (D(x, y, z + 1) + D(x + 1, y, z + 1));
      } else {
        div1 = quarter * (D(x, y, z) + D(x + 1, y, z) + D(x, y + 1, z) + D(x + 1, y + 1, z));
      }
      div1 = (R)a.hp.difmag * fmn((R)0, div1);
      double ul[5], ur[5];
      raw_cell(sl, ul);
      raw_cell(sr, ur);
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const R t = sizeof(R) == 8 ? (R)((double)(dt * (double)div1) * (ur[v] - ul[v]))
                                   : (R)(dt * (double)div1 * (ur[v] - ul[v]));
        F[v * NF + f] = zero_face ? (R)0 : scaled(fo[v]) + t;
      }
    } else {
#pragma unroll
      for (int v = 0; v < 5; v++) F[v * NF + f] = zero_face ? (R)0 : scaled(fo[v]);
    }
    if (PF) {
      // tmp: the face-normal velocity average and the internal-energy flux,
      // kept in this face's qm slots (read above, by this thread only)
      const R half = (R)0.5;
      qm[f] = zero_face ? (R)0 : scaled(half * (ql[1] + qr[1]));
      qm[NF + f] = zero_face ? (R)0 : scaled(fg[5]);
    }
  }
  cp_async_wait<0>();  // this thread's correction entries (E)
  __syncthreads();

  // ---- D. conservative update of active octs ----------------------------------
  double smax = 0.0, mass = 0.0, etot = 0.0, eint = 0.0;
  const double vol = a.dx * a.dx * a.dx;
  for (int it = tid; it < G::NCELL; it += NT) {
    // octs-major order: 8 consecutive threads update one oct (coalesced rows)
    const int o = it >> 3, ch = it & 7;
    const int ox = o % (TX / 2), oy = (o / (TX / 2)) % (TY / 2), oz = o / ((TX / 2) * (TY / 2));
    const int code = blk[(ox + 1) + BX * ((oy + 1) + BY * (oz + 1))];
    if (code < 0) continue;
    const int x = 2 * ox + (ch & 1), y = 2 * oy + ((ch >> 1) & 1), z = 2 * oz + (ch >> 2);
    const int fxl = x + (TX + 1) * (y + TY * z);
    const int fyl = NFX + x + TX * (y + (TY + 1) * z);
    const int fzl = NFX + NFY + x + TX * (y + TY * z);
    const int64_t dc = (int64_t)a.ncoarse + (int64_t)code * 8 + ch;
    double unv[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
      const R* Fv = F + v * NF;
      double un = a.fused ? __ldcg(a.uold + v * ncell + dc) : a.unew[v * ncell + dc];  // set_unew's value
      un = un + ((double)Fv[fxl] - (double)Fv[fxl + 1]);
      un = un + ((double)Fv[fyl] - (double)Fv[fyl + TX]);
      un = un + ((double)Fv[fzl] - (double)Fv[fzl + TX * TY]);
      a.unew[v * ncell + dc] = un;
      unv[v] = un;
    }
    if (PF) {
      // divu, then enew, each x then y then z, as unew (the fused form
      // starts them from set_unew's values: 0 and the internal energy of uold)
      const R* T1 = qm;
      const R* T2 = qm + NF;
      double dv, en;
      if (a.fused) {
        double uo[5];
#pragma unroll
        for (int v = 0; v < 5; v++) uo[v] = __ldcg(a.uold + v * ncell + dc);
        const double d = fmx(uo[0], a.hp.smallr);
        const double uu = uo[1] / d, vv = uo[2] / d, ww = uo[3] / d;
        dv = 0.0;
        en = uo[4] - 0.5 * d * (uu * uu + vv * vv + ww * ww);
      } else {
        dv = a.divu[dc];
        en = a.enew[dc];
      }
      dv = dv + ((double)T1[fxl] - (double)T1[fxl + 1]);
      dv = dv + ((double)T1[fyl] - (double)T1[fyl + TX]);
      dv = dv + ((double)T1[fzl] - (double)T1[fzl + TX * TY]);
      en = en + ((double)T2[fxl] - (double)T2[fxl + 1]);
      en = en + ((double)T2[fyl] - (double)T2[fyl + TX]);
      en = en + ((double)T2[fzl] - (double)T2[fzl + TX * TY]);
      a.divu[dc] = dv;
      a.enew[dc] = en;
    }
    if (a.fused == 1) {
      // courant_fine on the updated state (the next step's CFL condition);
      // the level minimum of dt_cell is dt_cell(maximum wave speed)
      const double ir = 1.0 / fmx(unv[0], a.hp.smallr);
      mass = mass + unv[0] * vol;
      etot = etot + unv[4] * vol;
      eint = eint + (unv[4] - 0.5 * (unv[1] * unv[1] + unv[2] * unv[2] + unv[3] * unv[3]) * ir) * vol;
      smax = fmx(smax, sizeof(R) == 8 ? cfl_speed(unv, a.hp) : cfl_speed_fast(unv, a.hp));
    }
  }
  if (a.fused == 1) {
    __shared__ double red[4][NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      smax = fmx(smax, __shfl_xor_sync(0xffffffffu, smax, o));
      mass += __shfl_xor_sync(0xffffffffu, mass, o);
      etot += __shfl_xor_sync(0xffffffffu, etot, o);
      eint += __shfl_xor_sync(0xffffffffu, eint, o);
    }
    if ((tid & 31) == 0) { red[0][tid >> 5] = smax; red[1][tid >> 5] = mass; red[2][tid >> 5] = etot; red[3][tid >> 5] = eint; }
    __syncthreads();
    if (tid == 0) {
      for (int k = 1; k < NT / 32; k++) { smax = fmx(smax, red[0][k]); mass += red[1][k]; etot += red[2][k]; eint += red[3][k]; }
      a.partial[(int64_t)tile * 4 + 0] = smax > 0.0 ? cfl_dt_from_speed(smax, a.dx, a.hp.courant_factor) : 1.0e300;
      a.partial[(int64_t)tile * 4 + 1] = mass;
      a.partial[(int64_t)tile * 4 + 2] = etot;
      a.partial[(int64_t)tile * 4 + 3] = eint;
    }
  }

  // ---- E. boundary fluxes for the fine-to-coarse correction --------------------
  if (a.tile_corr_off != nullptr) {
    const int n = corr_range[1] - corr_range[0];
    for (int it = tid; it < n * 20; it += NT) {
      const int i = it / 20, r = it % 20;
      const int ent = corr_ent[2 * i], slot = corr_ent[2 * i + 1];
      const int o = ent & 0xff, face = ent >> 8;   // face 0..5 = -x,+x,-y,+y,-z,+z
      const int ox = o % (TX / 2), oy = (o / (TX / 2)) % (TY / 2), oz = o / ((TX / 2) * (TY / 2));
      const int cc = r / 5, v = r % 5;
      const int d = face >> 1, side = face & 1;
      const int t1 = cc & 1, t2 = cc >> 1;
      int fidx;
      if (d == 0) { const int fx = 2 * ox + 2 * side; fidx = fx + (TX + 1) * ((2 * oy + t1) + TY * (2 * oz + t2)); }
      else if (d == 1) { const int fy = 2 * oy + 2 * side; fidx = NFX + (2 * ox + t1) + TX * (fy + (TY + 1) * (2 * oz + t2)); }
      else { const int fz = 2 * oz + 2 * side; fidx = NFX + NFY + (2 * ox + t1) + TX * ((2 * oy + t2) + TY * fz); }
      a.corr_flux[(int64_t)slot * 120 + face * 20 + r] = (double)F[v * NF + fidx];
      if (PF && v < 2) a.corr_tmp[(int64_t)slot * 48 + face * 8 + cc * 2 + v] = (double)qm[v * NF + fidx];
    }
  }
}

}  // namespace rb
