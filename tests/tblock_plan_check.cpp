// Invariants of the temporally blocked pass plan (gerjoii_b200/csrc/w_tblock_plan.h),
// checked on the host over many grids: every node owned exactly once; streaming
// tasks aligned, loading only fast rows and interior columns, owning only rows
// that are exact after D steps and none of the band frame's bottom rectangle;
// tiles no larger than their owned extent; interior tiles free of PML updates.
// Grid geometry as the radar plan sets it up (NX = pml_top + air + m + pml,
// NY = n + 2 pml, interior ranges of w_solve.m).  Prints "ok <cases>" or the
// first violation.
#include <cstdio>
#include <vector>

#include "w_tblock_plan.h"

using namespace gj;

static int fail(const char* what, int m, int n, int pml, int pt, int D, int G, int RC, int V, int st) {
  std::printf("FAIL %s: m=%d n=%d pml=%d pml_top=%d D=%d G=%d RC=%d V=%d stream=%d\n", what, m, n, pml, pt, D, G, RC,
              V, st);
  return 1;
}

int main() {
  const int ms[] = {24, 60, 130, 150, 290, 400, 517};
  const int ns[] = {40, 44, 100, 150, 401};
  int cases = 0;
  for (int m : ms)
    for (int n : ns)
      for (int pml : {8, 10, 30})
        for (int pt : {0, 1}) {
          const int ptop = pt ? pml : 0, air = pt ? 2 : 1;
          TbGeom g{};
          g.NX = ptop + air + m + pml;
          g.NY = n + 2 * pml;
          g.ei0 = ptop + 1; g.ei1 = g.NX - pml - 1; g.ej0 = pml + 1; g.ej1 = g.NY - pml - 1;
          g.hyi0 = ptop; g.hyi1 = g.NX - pml - 1; g.hxj0 = pml; g.hxj1 = g.NY - pml - 1;
          g.pml_top = ptop;
          g.bR0 = (g.NX - pml) / 4 * 4;
          for (int D = 1; D <= 4; ++D)
            for (int sh = 0; sh < 3; ++sh)
              for (int V : {4, 2})
                for (int st : {0, 1}) {
                  const int G = sh == 2 ? 4 : 2, RC = sh == 1 ? 64 : 32;
                  const TbPlan pl = tb_plan(g, D, G, RC, st != 0, V);
                  ++cases;
                  std::vector<int> own(size_t(g.NX + 1) * (g.NY + 1), 0);
                  auto mark = [&](int i, int j) { ++own[size_t(i) + size_t(j) * (g.NX + 1)]; };
                  const int RW = 32 * V;
                  for (const TbRowTask& t : pl.rows) {
                    if (t.R % V != 0) return fail("task row not vector aligned", m, n, pml, ptop, D, G, RC, V, st);
                    for (int I = (t.R > 0 ? t.R - 1 : 0); I <= t.R + RW; ++I)
                      if (!tb_fast_row(g, I)) return fail("task loads a row that is not fast", m, n, pml, ptop, D, G, RC, V, st);
                    const int ex_lo = t.R == 0 ? 0 : t.R + D - 1, ex_hi = t.R + RW - D + 1;
                    if (t.own_lo < ex_lo || t.own_hi > ex_hi || t.own_lo >= t.own_hi)
                      return fail("task owns rows that are not exact", m, n, pml, ptop, D, G, RC, V, st);
                    if (t.own_hi > g.bR0) return fail("task owns band-frame rows", m, n, pml, ptop, D, G, RC, V, st);
                    for (int i = t.own_lo; i < t.own_hi; ++i)
                      for (int j = pl.cs_lo; j <= pl.cs_hi; ++j) mark(i, j);
                  }
                  if (!pl.rows.empty()) {
                    // loaded columns [cs_lo - D, cs_hi + D]: Hx of the first, Ez of all
                    if (pl.cs_lo - D < g.hxj0 || pl.cs_lo - D + 1 < g.ej0 || pl.cs_hi + D - 1 > g.ej1)
                      return fail("streamed columns reach the PML", m, n, pml, ptop, D, G, RC, V, st);
                  }
                  const int TR = 32 * G - 2 * D, TC = RC - 2 * D;
                  bool seen_pml = false;
                  for (const TbTile& t : pl.tiles) {
                    if (t.tr < 1 || t.tc < 1 || t.tr > TR || t.tc > TC)
                      return fail("tile extent", m, n, pml, ptop, D, G, RC, V, st);
                    if (t.interior && seen_pml) return fail("interior tile after a PML tile", m, n, pml, ptop, D, G, RC, V, st);
                    seen_pml = seen_pml || !t.interior;
                    if (t.interior) {  // every node a step updates in the staged region is interior
                      for (int i = t.r0 - D; i < t.r0 - D + 32 * G; ++i)
                        for (int j = t.c0 - D; j < t.c0 - D + RC; ++j) {
                          if (i < 0 || i > g.NX || j < 0 || j > g.NY) continue;
                          const bool e = i >= 1 && i <= g.NX - 1 && j >= 1 && j <= g.NY - 1;
                          if (e && i > t.r0 - D && j > t.c0 - D && !(i >= g.ei0 && i <= g.ei1 && j >= g.ej0 && j <= g.ej1))
                            return fail("interior tile with a PML Ez node", m, n, pml, ptop, D, G, RC, V, st);
                        }
                    }
                    for (int i = t.r0; i < t.r0 + t.tr; ++i)
                      for (int j = t.c0; j < t.c0 + t.tc; ++j) {
                        if (i < 0 || i > g.NX || j < 0 || j > g.NY)
                          return fail("tile owns a node outside the grid", m, n, pml, ptop, D, G, RC, V, st);
                        mark(i, j);
                      }
                  }
                  for (int c : own)
                    if (c != 1) return fail("a node owned other than once", m, n, pml, ptop, D, G, RC, V, st);
                }
        }
  std::printf("ok %d\n", cases);
  return 0;
}
