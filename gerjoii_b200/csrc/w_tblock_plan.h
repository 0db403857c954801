// Host-side plan of a temporally blocked forward pass (w_tblock.cuh): which
// nodes the streaming interior tasks own and which the clipped tiles own.
// Plain C++ with no CUDA types, so the CPU tests compile it on its own and
// check its invariants over many grids.
//
// Streaming tasks load 32 V rows [R, R + 32 V) plus one halo row on each side,
// all of which must be fast rows (interior Ez rows, or the free top's Ez = 0
// row, that are also interior Hy rows); after D steps the rows
// [R + D - 1, R + 32 V - D] are exact (from row 0 when R = 0).  Tasks sit
// `stride` rows apart (R a multiple of V, for 16-byte vectors), each owning
// [R + D - 1, R + D - 1 + stride), and a last task aligned to the last
// eligible rows owns the rest of its exact rows.  The streamed rows stop above
// the band frame's bottom rectangle (row bR0), whose history the tiles write.
// Streamed columns: [ej0 + D - 1, ej1 - D + 1], so every loaded column is an
// interior column.  Every other node belongs to a clipped tile of at most
// TR x TC owned nodes (TR = 32 G - 2D, TC = RC - 2D), classified interior when
// every node that a step updates in its staged region (owned nodes + D halo)
// uses the interior formulas.
#pragma once
#include <algorithm>
#include <utility>
#include <vector>

namespace gj {

struct TbGeom {
  int NX, NY;                  // Yee nodes [0, NX] x [0, NY]
  int ei0, ei1, ej0, ej1;      // interior Ez nodes (w_solve.m:201)
  int hyi0, hyi1, hxj0, hxj1;  // interior Hy rows, interior Hx columns
  int pml_top;                 // 0: free top, row 0 is the Ez = 0 row
  int bR0;                     // first row of the band frame's bottom rectangle
};
struct TbRowTask { int R, own_lo, own_hi; };
struct TbTile { int r0, c0, tr, tc; bool interior; };
struct TbPlan {
  std::vector<TbRowTask> rows;  // streaming row tasks; empty: no streaming
  int cs_lo = 0, cs_hi = -1;    // streamed columns
  std::vector<TbTile> tiles;    // all other nodes, in launch order
};

inline bool tb_fast_row(const TbGeom& g, int I) {
  const bool e = (I >= g.ei0 && I <= g.ei1) || (I == 0 && g.pml_top == 0);
  return e && I >= g.hyi0 && I <= g.hyi1;
}

// D steps per pass; tiles stage 32 G rows x RC columns; streaming tasks hold V
// rows per lane (stream = false: tiles only).
inline TbPlan tb_plan(const TbGeom& g, int D, int G, int RC, bool stream, int V) {
  TbPlan pl;
  const int NX = g.NX, NY = g.NY;
  int rs_lo = 0, rs_hi = 0;
  if (stream) {
    const int RW = 32 * V;
    const int stride = V * ((RW + 2 - 2 * D) / V);
    auto eligible = [&](int R) {
      if (R + RW > NX - 1) return false;
      for (int I = std::max(R - 1, 0); I <= R + RW; ++I)
        if (!tb_fast_row(g, I)) return false;
      return true;
    };
    std::vector<TbRowTask> rows;
    int R = 0;
    while (R + RW <= NX - 1 && !eligible(R)) R += V;
    for (; eligible(R); R += stride) rows.push_back({R, R == 0 ? 0 : R + D - 1, R + D - 1 + stride});
    if (!rows.empty()) {
      int Rx = rows.back().R + stride - V;
      while (Rx > rows.back().R && !eligible(Rx)) Rx -= V;
      if (Rx > rows.back().R && Rx + RW - D + 1 > rows.back().own_hi)
        rows.push_back({Rx, rows.back().own_hi, Rx + RW - D + 1});
    }
    while (!rows.empty() && rows.back().own_hi > g.bR0) {
      rows.back().own_hi = g.bR0;
      if (rows.back().own_hi <= rows.back().own_lo) rows.pop_back();
      else break;
    }
    pl.cs_lo = g.ej0 + D - 1;
    pl.cs_hi = g.ej1 - D + 1;
    // task words pack rows and columns in 16 bits
    if (rows.empty() || pl.cs_hi < pl.cs_lo || NY >= 65536 || NX >= 65536) {
      pl.cs_hi = pl.cs_lo - 1;
    } else {
      pl.rows = rows;
      rs_lo = rows.front().own_lo;
      rs_hi = rows.back().own_hi;
    }
  }
  const int RR = 32 * G, TR = RR - 2 * D, TC = RC - 2 * D;
  std::vector<TbTile> ti, tp;
  auto tile_rect = [&](int a0, int a1, int b0, int b1) {
    for (int c0 = b0; c0 <= b1; c0 += TC)
      for (int r0 = a0; r0 <= a1; r0 += TR) {
        const int tr = std::min(TR, a1 - r0 + 1), tc = std::min(TC, b1 - c0 + 1);
        bool interior = true;
        for (int col = 0; col < RC && interior; ++col) {
          const int j = c0 - D + col;
          if (j < 0 || j > NY) continue;
          for (int row = 0; row < RR; ++row) {
            const int i = r0 - D + row;
            if (i < 0 || i > NX) continue;
            const bool hx = j <= NY - 1 && col < RC - 1, hy = i <= NX - 1 && row < RR - 1;
            const bool e = i >= 1 && i <= NX - 1 && j >= 1 && j <= NY - 1 && row >= 1 && col >= 1;
            if ((hx && !(j >= g.hxj0 && j <= g.hxj1)) || (hy && !(i >= g.hyi0 && i <= g.hyi1)) ||
                (e && !(i >= g.ei0 && i <= g.ei1 && j >= g.ej0 && j <= g.ej1))) {
              interior = false;
              break;
            }
          }
        }
        (interior ? ti : tp).push_back({r0, c0, tr, tc, interior});
      }
  };
  if (pl.rows.empty()) {
    tile_rect(0, NX, 0, NY);
  } else {
    if (rs_lo > 0) tile_rect(0, rs_lo - 1, 0, NY);
    if (rs_hi <= NX) tile_rect(rs_hi, NX, 0, NY);
    if (pl.cs_lo > 0) tile_rect(rs_lo, rs_hi - 1, 0, pl.cs_lo - 1);
    if (pl.cs_hi < NY) tile_rect(rs_lo, rs_hi - 1, pl.cs_hi + 1, NY);
  }
  pl.tiles = ti;  // interior tiles first, then PML tiles
  pl.tiles.insert(pl.tiles.end(), tp.begin(), tp.end());
  return pl;
}

}  // namespace gj
