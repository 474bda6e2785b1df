// e2d_ilu.cuh — the ILU(k) block preconditioner of the Newton-Krylov solve
// (Block_Preconditioner, NewtonKrylovSchwarz2D/Block_Preconditioner2D.h:
// 290-584 with BPKIT's BILUK, bpkit/src/BILUK.cc:55-205, and its symbolic
// factorization symbolic_ilu, bpkit/src/SparseUtil.cc:198).  Included by
// e2d_nks.cu inside its anonymous namespace, after the face Jacobian,
// normalisation and 4x4 inverse it shares with the block-Jacobi path.
//
// The reference builds, per solution block, a sparse matrix with one 4x4
// block per cell pair over ALL NCi x NCj cells (ghosts included): the
// first-order HLLE Jacobian on the five-point stencil for interior cells,
// identity rows for ghost cells, no coupling between the two.  BILUK then
// factors it with level-of-fill k in the natural cell order (i fastest) and
// inverts every diagonal block of U exactly (LP_INVERSE).
//
// The level-of-fill pattern depends on the ghost rows (a fill entry between
// two interior cells can be admitted by a path through ghost cells), so the
// symbolic factorization here runs on the full NCi x NCj pattern exactly as
// BPKIT does.  Numerically, every entry that couples an interior and a ghost
// cell is zero and stays zero through the factorization (the ghost rows are
// identity rows with zero off-diagonal blocks), so the device keeps only the
// interior rows and columns of that pattern: the same factors, without the
// ghost work.
//
// Device layout, one pattern shared by every block of the handle:
//   entries of interior row r (r = y * nci + x): row_ptr[r] .. row_ptr[r+1],
//   columns ascending, L part first (nlow[r] entries), then the diagonal,
//   then the rest of U; values vals[block][entry][16] (row-major 4x4) and
//   the inverted U diagonal dinv[block][row][16].
// Work lists: fop[fop_ptr[e] .. fop_ptr[e+1]] are the (target entry, U
// entry) pairs eliminating L entry e updates (BILUK.cc:122-132 in order);
// flev_* / blev_* are the rows by level of the forward (factorization and
// lower solve) and backward (upper solve) dependency graphs.
#pragma once
// (needs <map> and <vector>, included by e2d_nks.cu at file scope)

struct IluPattern {
  int nrow = 0, nnz = 0, nflev = 0, nblev = 0, maxrow = 0, maxops = 0, level = -1, nci = 0, ncj = 0;
  std::vector<int> row_ptr, nlow, col, fop_ptr, flev_ptr, flev_rows, blev_ptr, blev_rows, apos;
  std::vector<int2> fop;
  std::vector<int4> fdesc, bdesc, xdesc;
  std::vector<int2> xops;
};

struct IluDev {
  int nrow, nnz, nflev, nblev, maxrow, maxops;
  const int *row_ptr, *nlow, *col, *fop_ptr;
  const int2* fop;
  const int *flev_ptr, *flev_rows, *blev_ptr, *blev_rows, *apos;
  const int4 *fdesc, *bdesc;  // per level-ordered row: (row, first entry, end entry, 0)
  const int4* xdesc;          // factorization, level order: (row, first entry, L entries, entries)
  const int2* xops;           // factorization, level order: the row's elimination list range
  double* vals;
  double* dinv;
  double* work;  // [nblk][nrow][4] when a block's vector does not fit shared memory
};

// Level-of-fill pattern of the NCi x NCj five-point block matrix, restricted
// to interior cells.  Levels follow symbolic_ilu: A's entries have level 0,
// eliminating column k of row i offers column j of U(k) the level
// lev(i,k) + lev(k,j) + 1, kept when <= k_fill or when j is already in the
// row (then the minimum).  Returns false if the pattern is too large.
inline bool ilu_pattern(int nci, int ncj, int k_fill, IluPattern& P) {
  const int NCi = nci + 4, NCj = ncj + 4, n = NCi * NCj;
  std::vector<std::vector<std::pair<int, int>>> Ufull(n);  // (col, level), diagonal first
  std::vector<std::vector<int>> full(n);                     // row pattern, ascending
  std::map<int, int> row;
  for (int i = 0; i < n; ++i) {
    row.clear();
    // Get_Block_Index (Block_Preconditioner2D.h:180-188): N, E, C, W, S
    if (i - NCi >= 0) row[i - NCi] = 0;
    if (i % NCi != 0) row[i - 1] = 0;
    row[i] = 0;
    if ((i + 1) % NCi != 0) row[i + 1] = 0;
    if (i + NCi < n) row[i + NCi] = 0;
    for (auto it = row.begin(); it != row.end() && it->first < i; ++it) {
      const int k = it->first, lk = it->second;
      for (size_t q = 1; q < Ufull[k].size(); ++q) {
        const int j = Ufull[k][q].first, nl = lk + Ufull[k][q].second + 1;
        auto f = row.find(j);
        if (f != row.end()) {
          if (nl < f->second) f->second = nl;
        } else if (nl <= k_fill) {
          row.emplace(j, nl);
        }
      }
    }
    for (const auto& e : row) {
      full[i].push_back(e.first);
      if (e.first >= i) Ufull[i].emplace_back(e.first, e.second);
    }
  }
  auto interior = [&](int f) {
    const int x = f % NCi, y = f / NCi;
    return (x >= 2 && x < NCi - 2 && y >= 2 && y < NCj - 2) ? (y - 2) * nci + (x - 2) : -1;
  };
  const int nr = nci * ncj;
  P = IluPattern();
  P.nrow = nr;
  P.level = k_fill;
  P.nci = nci;
  P.ncj = ncj;
  P.row_ptr.assign(nr + 1, 0);
  P.nlow.assign(nr, 0);
  for (int f = 0; f < n; ++f) {
    const int r = interior(f);
    if (r < 0) continue;
    for (int cf : full[f]) {
      const int c = interior(cf);
      if (c < 0) continue;
      P.col.push_back(c);
      if (c < r) ++P.nlow[r];
    }
    P.row_ptr[r + 1] = int(P.col.size());
    P.maxrow = std::max(P.maxrow, P.row_ptr[r + 1] - P.row_ptr[r]);
    if (P.col.size() > (size_t(1) << 26)) return false;
  }
  P.nnz = int(P.col.size());
  auto find = [&](int r, int c) {
    for (int e = P.row_ptr[r]; e < P.row_ptr[r + 1]; ++e)
      if (P.col[e] == c) return e;
    return -1;
  };
  // elimination work lists
  P.fop_ptr.assign(P.nnz + 1, 0);
  for (int r = 0; r < nr; ++r) {
    for (int e = P.row_ptr[r]; e < P.row_ptr[r + 1]; ++e) {
      if (e < P.row_ptr[r] + P.nlow[r]) {
        const int id = P.col[e];
        for (int q = P.row_ptr[id] + P.nlow[id] + 1; q < P.row_ptr[id + 1]; ++q) {
          const int t = find(r, P.col[q]);
          if (t >= 0) P.fop.push_back(make_int2(t, q));
        }
      }
      P.fop_ptr[e + 1] = int(P.fop.size());
    }
    P.maxops = std::max(P.maxops, P.fop_ptr[P.row_ptr[r + 1]] - P.fop_ptr[P.row_ptr[r]]);
  }
  // level schedules
  std::vector<int> lev(nr, 0);
  int maxl = 0;
  for (int r = 0; r < nr; ++r) {
    int l = 0;
    for (int e = P.row_ptr[r]; e < P.row_ptr[r] + P.nlow[r]; ++e) l = std::max(l, lev[P.col[e]] + 1);
    lev[r] = l;
    maxl = std::max(maxl, l);
  }
  P.nflev = maxl + 1;
  P.flev_ptr.assign(P.nflev + 1, 0);
  for (int r = 0; r < nr; ++r) ++P.flev_ptr[lev[r] + 1];
  for (int l = 0; l < P.nflev; ++l) P.flev_ptr[l + 1] += P.flev_ptr[l];
  P.flev_rows.assign(nr, 0);
  {
    std::vector<int> fill(P.flev_ptr.begin(), P.flev_ptr.end() - 1);
    for (int r = 0; r < nr; ++r) P.flev_rows[fill[lev[r]]++] = r;
  }
  maxl = 0;
  for (int r = nr - 1; r >= 0; --r) {
    int l = 0;
    for (int e = P.row_ptr[r] + P.nlow[r] + 1; e < P.row_ptr[r + 1]; ++e) l = std::max(l, lev[P.col[e]] + 1);
    lev[r] = l;
    maxl = std::max(maxl, l);
  }
  P.nblev = maxl + 1;
  P.blev_ptr.assign(P.nblev + 1, 0);
  for (int r = 0; r < nr; ++r) ++P.blev_ptr[lev[r] + 1];
  for (int l = 0; l < P.nblev; ++l) P.blev_ptr[l + 1] += P.blev_ptr[l];
  P.blev_rows.assign(nr, 0);
  {
    std::vector<int> fill(P.blev_ptr.begin(), P.blev_ptr.end() - 1);
    for (int r = nr - 1; r >= 0; --r) P.blev_rows[fill[lev[r]]++] = r;
  }
  // row descriptors in level order: the L part (forward), the U part past
  // the diagonal (backward)
  P.fdesc.resize(nr);
  P.bdesc.resize(nr);
  P.xdesc.resize(nr);
  P.xops.resize(nr);
  for (int q = 0; q < nr; ++q) {
    const int i = P.flev_rows[q], k = P.blev_rows[q];
    P.fdesc[q] = make_int4(i, P.row_ptr[i], P.row_ptr[i] + P.nlow[i], 0);
    P.bdesc[q] = make_int4(k, P.row_ptr[k] + P.nlow[k] + 1, P.row_ptr[k + 1], 0);
    P.xdesc[q] = make_int4(i, P.row_ptr[i], P.nlow[i], P.row_ptr[i + 1] - P.row_ptr[i]);
    P.xops[q] = make_int2(P.fop_ptr[P.row_ptr[i]], P.fop_ptr[P.row_ptr[i] + P.nlow[i]]);
  }
  // where cell c's column blocks go: its diagonal, then the rows of the
  // cells below (j-1), above (j+1), left (i-1), right (i+1) — the reference's
  // NORTH, SOUTH, EAST, WEST blocks (Block_Preconditioner2D.h:209-231)
  P.apos.assign(5 * size_t(nr), -1);
  for (int r = 0; r < nr; ++r) {
    const int x = r % nci, y = r / nci;
    P.apos[5 * r + 0] = P.row_ptr[r] + P.nlow[r];
    if (y > 0) P.apos[5 * r + 1] = find(r - nci, r);
    if (y < ncj - 1) P.apos[5 * r + 2] = find(r + nci, r);
    if (x > 0) P.apos[5 * r + 3] = find(r - 1, r);
    if (x < nci - 1) P.apos[5 * r + 4] = find(r + 1, r);
  }
  return true;
}

__device__ __forceinline__ double cell_area(const Blocks& B, int b, int i, int j) {
  double xc, yc, A;
  quad_centroid(nodeX(B, b, i, j), nodeY(B, b, i, j), nodeX(B, b, i + 1, j), nodeY(B, b, i + 1, j),
                nodeX(B, b, i + 1, j + 1), nodeY(B, b, i + 1, j + 1), nodeX(B, b, i, j + 1), nodeY(B, b, i, j + 1),
                xc, yc, A);
  return A;
}

// Update_Jacobian_and_Preconditioner's matrix (Block_Preconditioner2D.h:
// 352-460): per interior cell, Implicit_Euler (-I/dt on the diagonal) plus,
// for the first-order HLLE Jacobian, the four face blocks F: the diagonal
// gains (F_N + F_S + F_E + F_W) / A, the neighbour rows -F / A(neighbour)
// (dropped where the neighbour is a ghost cell); every block normalized.
// vals must be zero beforehand (fill entries start at zero).
__global__ void __launch_bounds__(128) ilu_assemble_kernel(Blocks B, IluDev D, double ao, int hlle) {
  const long long n = (long long)B.nblk * B.nci * B.ncj;
  const int per = B.nci * B.ncj;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int b = int(q / per), r = int(q % per);
    if (B.case_active && !B.case_active[case_id(B, b)]) continue;
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    const size_t c = cell_sc(B, b, j, i);
    double* V = D.vals + (size_t(b) * D.nnz) * 16;
    const int* ap = D.apos + 5 * size_t(r);
    const double lhs = 1.0 / B.dt[c];
    double m[4][4];
    if (!hlle) {  // Source_Terms_Only: -I / dt alone
#pragma unroll
      for (int rr = 0; rr < 4; ++rr)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) m[rr][cc] = rr == cc ? -lhs : 0.0;
      normalize_block(m, ao);
#pragma unroll
      for (int rr = 0; rr < 4; ++rr)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) V[16 * size_t(ap[0]) + 4 * rr + cc] = m[rr][cc];
      continue;
    }
    const PState<double> wc = ldW(B, b, i, j);
    double F[4][4][4];
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
      for (int rr = 0; rr < 4; ++rr)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) F[f][rr][cc] = 0.0;
    double nx, ny;
    nfaceN(B, b, i, j - 1, nx, ny);
    face_jacobian(wc, ldW(B, b, i, j - 1), nx, ny, glen(B, b, i, j, i + 1, j), B.g, B.gm1, B.gm1i, F[0]);
    nfaceS(B, b, i, j + 1, nx, ny);
    face_jacobian(wc, ldW(B, b, i, j + 1), nx, ny, glen(B, b, i, j + 1, i + 1, j + 1), B.g, B.gm1, B.gm1i, F[1]);
    nfaceE(B, b, i - 1, j, nx, ny);
    face_jacobian(wc, ldW(B, b, i - 1, j), nx, ny, glen(B, b, i, j, i, j + 1), B.g, B.gm1, B.gm1i, F[2]);
    nfaceW(B, b, i + 1, j, nx, ny);
    face_jacobian(wc, ldW(B, b, i + 1, j), nx, ny, glen(B, b, i + 1, j, i + 1, j + 1), B.g, B.gm1, B.gm1i, F[3]);
    const double A = cell_area(B, b, i, j);
#pragma unroll
    for (int rr = 0; rr < 4; ++rr)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) {
        const double s = ((F[0][rr][cc] + F[1][rr][cc]) + F[2][rr][cc]) + F[3][rr][cc];
        m[rr][cc] = (rr == cc ? -lhs : 0.0) + s / A;
      }
    normalize_block(m, ao);
#pragma unroll
    for (int rr = 0; rr < 4; ++rr)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) V[16 * size_t(ap[0]) + 4 * rr + cc] = m[rr][cc];
    const int ni[4] = {i, i, i - 1, i + 1}, nj[4] = {j - 1, j + 1, j, j};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const int pos = ap[1 + f];
      if (pos < 0) continue;
      const double An = cell_area(B, b, ni[f], nj[f]);
#pragma unroll
      for (int rr = 0; rr < 4; ++rr)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) m[rr][cc] = (-F[f][rr][cc]) / An;
      normalize_block(m, ao);
#pragma unroll
      for (int rr = 0; rr < 4; ++rr)
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) V[16 * size_t(pos) + 4 * rr + cc] = m[rr][cc];
    }
  }
}

constexpr int ILU_THREADS = 256;
// the solves: 32 rows of a level at a time (4 threads per row); fewer idle
// warps share the schedulers with the ones on the critical path
constexpr int ILU_APPLY_THREADS = 128;

// BILUK::setup's numeric factorization (BILUK.cc:85-150), one CTA per
// block, rows level by level; a row is worked by 16 threads, one per element
// of the 4x4 blocks, in shared memory: the row's blocks, columns and
// elimination work list are staged per 16-thread group (D.maxrow entries,
// D.maxops updates).  For each L entry in column order: mult = L * inv(D_id)
// (kept as the L factor), then every pattern entry t of the row that U(id)
// reaches gets t -= mult * U(id, .); the finished row goes back to global
// memory and its diagonal block is inverted.  Products accumulate in the
// order of the netlib dgemm loops BPKIT calls.
constexpr int ILU_OPS_CHUNK = 8;

__global__ void __launch_bounds__(ILU_THREADS) ilu_factor_kernel(Blocks B, IluDev D) {
  extern __shared__ double rsh[];
  const int b = blockIdx.x;
  if (B.case_active && !B.case_active[case_id(B, b)]) return;
  double* V = D.vals + (size_t(b) * D.nnz) * 16;
  double* Di = D.dinv + (size_t(b) * D.nrow) * 16;
  const int grp = threadIdx.x >> 4, lane = threadIdx.x & 15, r = lane >> 2, c = lane & 3;
  const unsigned gmask = 0xFFFFu << (threadIdx.x & 16);
  __shared__ double msh[ILU_THREADS];
  double* mg = msh + (threadIdx.x & ~15);
  // per group: blocks [maxrow][16], columns [maxrow], op offsets [maxrow + 2], ops [maxops]
  const size_t per = 16 * size_t(D.maxrow) * sizeof(double) + (2 * size_t(D.maxrow) + 2) * sizeof(int) +
                     size_t(D.maxops) * sizeof(int2);
  unsigned char* gbase = reinterpret_cast<unsigned char*>(rsh) + size_t(grp) * per;
  double* row = reinterpret_cast<double*>(gbase);
  int* gcol = reinterpret_cast<int*>(row + 16 * D.maxrow);
  int* gfp = gcol + D.maxrow;
  int2* gops = reinterpret_cast<int2*>(gfp + D.maxrow + 2);
  __shared__ int lev_ptr[2];
  for (int L = 0; L < D.nflev; ++L) {
    if (threadIdx.x < 2) lev_ptr[threadIdx.x] = D.flev_ptr[L + threadIdx.x];
    __syncthreads();
    const int q0 = lev_ptr[0], q1 = lev_ptr[1];
    for (int q = q0 + grp; q < q1; q += ILU_THREADS / 16) {
      const int4 xd = D.xdesc[q];
      const int2 xo = D.xops[q];
      const int i = xd.x, e0 = xd.y, nL = xd.z, nE = xd.w;
      const int ob = xo.x, oe = xo.y;
      for (int e = 0; e < nE; ++e) row[16 * e + lane] = V[16 * size_t(e0 + e) + lane];
      for (int t = lane; t < nE; t += 16) gcol[t] = D.col[e0 + t];
      for (int t = lane; t <= nL; t += 16) gfp[t] = D.fop_ptr[e0 + t] - ob;
      for (int t = lane; t < oe - ob; t += 16) {
        const int2 o = D.fop[ob + t];
        gops[t] = make_int2(o.x - e0, o.y);
      }
      __syncwarp(gmask);
      double dn[4] = {0.0, 0.0, 0.0, 0.0};
      if (nL > 0) {
        const double* Dd = Di + 16 * size_t(gcol[0]);
#pragma unroll
        for (int l = 0; l < 4; ++l) dn[l] = Dd[4 * l + c];
      }
      for (int le = 0; le < nL; ++le) {
        const double d0 = dn[0], d1 = dn[1], d2 = dn[2], d3 = dn[3];
        if (le + 1 < nL) {  // the next L entry's inverted diagonal, a step ahead
          const double* Dd = Di + 16 * size_t(gcol[le + 1]);
#pragma unroll
          for (int l = 0; l < 4; ++l) dn[l] = Dd[4 * l + c];
        }
        double* Le = row + 16 * le;
        __syncwarp(gmask);
        const double a0 = Le[4 * r + 0], a1 = Le[4 * r + 1], a2 = Le[4 * r + 2], a3 = Le[4 * r + 3];
        double m = 0.0;
        m = m + d0 * a0;
        m = m + d1 * a1;
        m = m + d2 * a2;
        m = m + d3 * a3;
        mg[lane] = m;
        __syncwarp(gmask);
        Le[lane] = m;
        const double m0 = mg[4 * r + 0], m1 = mg[4 * r + 1], m2 = mg[4 * r + 2], m3 = mg[4 * r + 3];
        // the updates of one L entry hit distinct entries: a chunk at a
        // time, its U loads issued together
        for (int o = gfp[le]; o < gfp[le + 1]; o += ILU_OPS_CHUNK) {
          const int n = min(ILU_OPS_CHUNK, gfp[le + 1] - o);
          double u[ILU_OPS_CHUNK][4];
#pragma unroll
          for (int kk = 0; kk < ILU_OPS_CHUNK; ++kk)
            if (kk < n) {
              const double* U = V + 16 * size_t(gops[o + kk].y);
              u[kk][0] = U[0 + c]; u[kk][1] = U[4 + c]; u[kk][2] = U[8 + c]; u[kk][3] = U[12 + c];
            }
#pragma unroll
          for (int kk = 0; kk < ILU_OPS_CHUNK; ++kk)
            if (kk < n) {
              double* t = row + 16 * gops[o + kk].x + lane;
              double acc = *t;
              acc = acc + (-u[kk][0]) * m0;
              acc = acc + (-u[kk][1]) * m1;
              acc = acc + (-u[kk][2]) * m2;
              acc = acc + (-u[kk][3]) * m3;
              *t = acc;
            }
        }
      }
      __syncwarp(gmask);
      for (int e = 0; e < nE; ++e) V[16 * size_t(e0 + e) + lane] = row[16 * e + lane];
      if (lane == 0) {
        double a[4][4];
#pragma unroll
        for (int rr = 0; rr < 4; ++rr)
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) a[rr][cc] = row[16 * nL + 4 * rr + cc];
        if (!invert4(a)) set_status(B.status, 3, int(cell_sc(B, b, NG + i / B.nci, NG + i % B.nci)));
#pragma unroll
        for (int rr = 0; rr < 4; ++rr)
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) Di[16 * size_t(i) + 4 * rr + cc] = a[rr][cc];
      }
      __syncwarp(gmask);
    }
    __syncthreads();
  }
}

// size of ilu_factor_kernel's dynamic shared memory
inline size_t ilu_factor_smem_bytes(const IluPattern& P) {
  return size_t(ILU_THREADS / 16) * (16 * size_t(P.maxrow) * sizeof(double) +
                                     (2 * size_t(P.maxrow) + 2) * sizeof(int) + size_t(P.maxops) * sizeof(int2));
}

// acc - sum over entries e0..e1 (in order) of block(e) row k . y(col(e)):
// one row of a triangular solve, the loads of four entries issued together.
__device__ __forceinline__ double row_solve(const double* __restrict__ V, const double* y, const int* __restrict__ col,
                                            int e0, int e1, int k, double acc) {
  int e = e0;
  for (; e + 4 <= e1; e += 4) {
    double a[4][4], w[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double* Bq = V + 16 * size_t(e + q) + 4 * k;
      const double* yq = y + 4 * col[e + q];
#pragma unroll
      for (int l = 0; l < 4; ++l) { a[q][l] = Bq[l]; w[q][l] = yq[l]; }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int l = 0; l < 4; ++l) acc = acc + (-w[q][l]) * a[q][l];
  }
  for (; e < e1; ++e) {
    const double* Bq = V + 16 * size_t(e) + 4 * k;
    const double* yq = y + 4 * col[e];
    acc = acc + (-yq[0]) * Bq[0];
    acc = acc + (-yq[1]) * Bq[1];
    acc = acc + (-yq[2]) * Bq[2];
    acc = acc + (-yq[3]) * Bq[3];
  }
  return acc;
}

// A row of a triangular solve whose first four entries (values, columns
// and, for the upper solve, the inverted diagonal block) are loaded a level
// ahead, while the level before it is still being solved.
struct RowPre {
  int i, e, end;
  int col[4];
  double a[4][4];
  double dd[4];
};

template <bool BACK>
__device__ __forceinline__ void row_prefetch(const int4* desc, const int* lp, int L, int nlev, int grp, int k,
                                             const double* __restrict__ V, const double* __restrict__ Di,
                                             const int* __restrict__ col, RowPre& p) {
  p.i = -1;
  if (L >= nlev) return;
  const int q = lp[L] + grp;
  if (q >= lp[L + 1]) return;
  const int4 d = desc[q];
  p.i = d.x; p.e = d.y; p.end = d.z;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    if (d.y + m < d.z) {
      p.col[m] = col[d.y + m];
      const double* Bq = V + 16 * size_t(d.y + m) + 4 * k;
#pragma unroll
      for (int l = 0; l < 4; ++l) p.a[m][l] = Bq[l];
    }
  }
  if (BACK) {
    const double* Dd = Di + 16 * size_t(d.x) + 4 * k;
#pragma unroll
    for (int l = 0; l < 4; ++l) p.dd[l] = Dd[l];
  }
}

__device__ __forceinline__ double row_finish(const RowPre& p, const double* __restrict__ V, const double* y,
                                             const int* __restrict__ col, int k, double acc) {
#pragma unroll
  for (int m = 0; m < 4; ++m)
    if (p.e + m < p.end) {
      const double* yq = y + 4 * p.col[m];
#pragma unroll
      for (int l = 0; l < 4; ++l) acc = acc + (-yq[l]) * p.a[m][l];
    }
  if (p.end > p.e + 4) acc = row_solve(V, y, col, p.e + 4, p.end, k, acc);
  return acc;
}

// BILUK::apply (BILUK.cc:152-205): z = inv(U) inv(L) v on the interior
// cells of each block, v and z GMRES vectors ([nblk][NCj][NCi][4], ghosts
// zero and left alone).  One CTA per block, 4 threads per row (one per
// variable), rows level by level; the block's vector is worked in shared
// memory (SHARED) or in D.work.
template <bool SHARED>
__global__ void __launch_bounds__(ILU_APPLY_THREADS) ilu_apply_kernel(Blocks B, IluDev D, const double* __restrict__ v,
                                                                double* __restrict__ z) {
  extern __shared__ double ysh[];
  const int b = blockIdx.x;
  if (B.case_active && !B.case_active[case_id(B, b)]) return;
  const double* V = D.vals + (size_t(b) * D.nnz) * 16;
  const double* Di = D.dinv + (size_t(b) * D.nrow) * 16;
  // shared: the block's vector, the row descriptors in level order and the
  // level offsets (everything a level reads except the factor values)
  double* y = SHARED ? ysh : D.work + size_t(b) * D.nrow * 4;
  const int4* fdesc = D.fdesc;
  const int4* bdesc = D.bdesc;
  const int* flp = D.flev_ptr;
  const int* blp = D.blev_ptr;
  if (SHARED) {
    int4* fd = reinterpret_cast<int4*>(ysh + 4 * size_t(D.nrow));
    int4* bd = fd + D.nrow;
    int* fl = reinterpret_cast<int*>(bd + D.nrow);
    int* bl = fl + D.nflev + 1;
    for (int t = threadIdx.x; t < D.nrow; t += ILU_APPLY_THREADS) { fd[t] = D.fdesc[t]; bd[t] = D.bdesc[t]; }
    for (int t = threadIdx.x; t <= D.nflev; t += ILU_APPLY_THREADS) fl[t] = D.flev_ptr[t];
    for (int t = threadIdx.x; t <= D.nblev; t += ILU_APPLY_THREADS) bl[t] = D.blev_ptr[t];
    fdesc = fd; bdesc = bd; flp = fl; blp = bl;
  }
  const size_t base = size_t(b) * B.NCj * B.NCi;
  for (int t = threadIdx.x; t < 4 * D.nrow; t += ILU_APPLY_THREADS) {
    const int r = t >> 2;
    y[t] = v[4 * (base + size_t(NG + r / B.nci) * B.NCi + NG + r % B.nci) + (t & 3)];
  }
  __syncthreads();
  const int grp = threadIdx.x >> 2, k = threadIdx.x & 3;
  const unsigned qmask = 0xFu << (threadIdx.x & 28);
  // forward solve with the unit lower factor (level 0 rows have no L part);
  // a group's first row of each level is prefetched during the level before
  RowPre cur, nxt;
  row_prefetch<false>(fdesc, flp, 1, D.nflev, grp, k, V, Di, D.col, cur);
  for (int L = 1; L < D.nflev; ++L) {
    row_prefetch<false>(fdesc, flp, L + 1, D.nflev, grp, k, V, Di, D.col, nxt);
    if (cur.i >= 0) y[4 * cur.i + k] = row_finish(cur, V, y, D.col, k, y[4 * cur.i + k]);
    for (int q = flp[L] + grp + ILU_APPLY_THREADS / 4; q < flp[L + 1]; q += ILU_APPLY_THREADS / 4) {
      const int4 d = fdesc[q];
      y[4 * d.x + k] = row_solve(V, y, D.col, d.y, d.z, k, y[4 * d.x + k]);
    }
    __syncthreads();
    cur = nxt;
  }
  // backward solve with U, then the inverted diagonal block
  row_prefetch<true>(bdesc, blp, 0, D.nblev, grp, k, V, Di, D.col, cur);
  for (int L = 0; L < D.nblev; ++L) {
    row_prefetch<true>(bdesc, blp, L + 1, D.nblev, grp, k, V, Di, D.col, nxt);
    if (cur.i >= 0) {
      const int i = cur.i;
      y[4 * i + k] = row_finish(cur, V, y, D.col, k, y[4 * i + k]);
      __syncwarp(qmask);
      double x = 0.0;
      x = x + y[4 * i + 0] * cur.dd[0];
      x = x + y[4 * i + 1] * cur.dd[1];
      x = x + y[4 * i + 2] * cur.dd[2];
      x = x + y[4 * i + 3] * cur.dd[3];
      __syncwarp(qmask);
      y[4 * i + k] = x;
    }
    for (int q = blp[L] + grp + ILU_APPLY_THREADS / 4; q < blp[L + 1]; q += ILU_APPLY_THREADS / 4) {
      const int4 d = bdesc[q];
      const double* Dd = Di + 16 * size_t(d.x) + 4 * k;
      const double d0 = Dd[0], d1 = Dd[1], d2 = Dd[2], d3 = Dd[3];
      y[4 * d.x + k] = row_solve(V, y, D.col, d.y, d.z, k, y[4 * d.x + k]);
      __syncwarp(qmask);
      double x = 0.0;
      x = x + y[4 * d.x + 0] * d0;
      x = x + y[4 * d.x + 1] * d1;
      x = x + y[4 * d.x + 2] * d2;
      x = x + y[4 * d.x + 3] * d3;
      __syncwarp(qmask);
      y[4 * d.x + k] = x;
    }
    __syncthreads();
    cur = nxt;
  }
  for (int t = threadIdx.x; t < 4 * D.nrow; t += ILU_APPLY_THREADS) {
    const int r = t >> 2;
    z[4 * (base + size_t(NG + r / B.nci) * B.NCi + NG + r % B.nci) + (t & 3)] = y[t];
  }
}
