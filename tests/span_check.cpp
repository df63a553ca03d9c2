// Host check of the row spans (tomo_span.cuh): for random triangles of
// several shapes, every pixel of the bounding box that the kernels' float
// pre-reject passes must lie inside its column's span.  The pre-reject is
// restated here with the kernels' float operations in their order (IEEE
// single precision, no contraction).  Prints one line:
// "triangles T pixels P passed Q span_items S box_items B violations V".
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cmath>
#include <random>

#include "../tomo_shell2026_b200/csrc/tomo_span.cuh"

using tomo::SpanTri;

static float pix_center(int x, float half) { return ((float)x + 0.001f) + half; }
static float dot2(float ax, float ay, float bx, float by) { return ((ax * bx) + (ay * by)) + 0.0f; }

struct Counts { long long tris = 0, pixels = 0, passed = 0, span_items = 0, box_items = 0, violations = 0; };

static void check(float ax, float ay, float bx, float by, float cx, float cy, float half, Counts& n)
{
  const int x0 = (int)std::trunc(std::fmin(std::fmin(ax, bx), cx));
  const int y0 = (int)std::trunc(std::fmin(std::fmin(ay, by), cy));
  const int x1 = (int)std::trunc(std::fmax(std::fmax(ax, bx), cx));
  const int y1 = (int)std::trunc(std::fmax(std::fmax(ay, by), cy));
  const int ylen = y1 - y0 + 1;
  const float e0x = bx - ax, e0y = by - ay, e1x = cx - ax, e1y = cy - ay;
  const float d00 = dot2(e0x, e0y, e0x, e0y), d01 = dot2(e0x, e0y, e1x, e1y), d11 = dot2(e1x, e1y, e1x, e1y);
  const float denom = (d00 * d11) - (d01 * d01);
  const float ad = denom >= 0.0f ? denom : -denom;
  if (!(ad > 0.001f)) return;   // the walk skips these triangles
  const bool dpos = denom > 0.0f;
  const float rlo = -0.002f * ad, rvhi = 1.002f * ad, rwhi = 1.004f * ad, ruhi = 1.003f * ad;
  const SpanTri T = tomo::span_setup(ax, ay, e0x, e0y, e1x, e1y, d00, d01, d11, dpos, rlo, ruhi, x0, x1, y0, ylen,
                                     half);
  n.tris++;
  for (int x = x0; x <= x1; x++) {
    const float px = pix_center(x, half);
    int lo = y0, hi = y1;   // triangles without spans walk the whole box
    if (T.ok) tomo::span_rows(T, px, y0, ylen, lo, hi);
    if (hi >= lo) n.span_items += hi - lo + 1;
    n.box_items += ylen;
    const float ex0 = (px - ax) * e0x, ex1 = (px - ax) * e1x;
    for (int y = y0; y <= y1; y++) {
      const float e2y = pix_center(y, half) - ay;
      const float d20 = ex0 + (e2y * e0y);
      const float d21 = ex1 + (e2y * e1y);
      const float vn = (d11 * d20) - (d01 * d21);
      const float wn = (d00 * d21) - (d01 * d20);
      const float vs = dpos ? vn : -vn, ws = dpos ? wn : -wn;
      const bool pass = !(vs < rlo || vs > rvhi || ws < rlo || ws > rwhi || (vs + ws) > ruhi);
      n.pixels++;
      if (!pass) continue;
      n.passed++;
      if (y < lo || y > hi) {
        if (n.violations < 10)
          std::printf("violation: tri (%.9g %.9g) (%.9g %.9g) (%.9g %.9g) half %g column %d row %d span [%d, %d]\n",
                      ax, ay, bx, by, cx, cy, half, x, y, lo, hi);
        n.violations++;
      }
    }
  }
}

int main(int argc, char** argv)
{
  const long long per_kind = argc > 1 ? std::atoll(argv[1]) : 100000;
  const unsigned seed = argc > 2 ? (unsigned)std::atoi(argv[2]) : 1u;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  auto uf = [&](double a, double b) { return (float)(a + (b - a) * U(rng)); };
  const float halves[] = {0.5f, 0.25f, 1.0f, 0.125f};
  Counts n;
  for (long long i = 0; i < per_kind; i++) {
    const float half = halves[i & 3];
    const float ox = uf(0.0, 4000.0), oy = uf(0.0, 4000.0);
    // small triangles, a few pixels across
    check(ox + uf(0, 4), oy + uf(0, 4), ox + uf(0, 4), oy + uf(0, 4), ox + uf(0, 4), oy + uf(0, 4), half, n);
    // medium and large (up to the 63-row span limit and beyond)
    const double s = (i % 7 == 0) ? 200.0 : 40.0;
    check(ox + uf(0, s), oy + uf(0, s), ox + uf(0, s), oy + uf(0, s), ox + uf(0, s), oy + uf(0, s), half, n);
    // slivers: a long edge and a third vertex very near it
    {
      const float ax = ox, ay = oy, bx = ox + uf(-30, 30), by = oy + uf(-30, 30);
      const float t = uf(0, 1), d = (float)std::ldexp(U(rng), -(int)(U(rng) * 20));
      const float cx = ax + t * (bx - ax) - d * (by - ay) * 0.01f, cy = ay + t * (by - ay) + d * (bx - ax) * 0.01f;
      check(ax, ay, bx, by, cx, cy, half, n);
    }
    // axis-aligned edges and vertices on pixel centres and pixel edges
    {
      const float bx0 = std::floor(ox), by0 = std::floor(oy);
      const float fx = (i % 3 == 0) ? 0.0f : (i % 3 == 1 ? 0.001f + half : 0.5f);
      const float w = (float)(1 + (int)(U(rng) * 6)), h = (float)(1 + (int)(U(rng) * 6));
      if (i & 4) check(bx0 + fx, by0 + fx, bx0 + fx + w, by0 + fx, bx0 + fx, by0 + fx + h, half, n);
      else check(bx0 + fx + w, by0 + fx + h, bx0 + fx, by0 + fx + h, bx0 + fx + w, by0 + fx, half, n);
    }
    // near-degenerate (almost collinear) small triangles
    {
      const float ax = ox + uf(0, 3), ay = oy + uf(0, 3), bx = ax + uf(-3, 3), by = ay + uf(-3, 3);
      const float e = (float)std::ldexp(1.0, -(int)(8 + U(rng) * 14));
      check(ax, ay, bx, by, ax + 2.0f * (bx - ax) + e, ay + 2.0f * (by - ay) - e, half, n);
    }
  }
  std::printf("triangles %lld pixels %lld passed %lld span_items %lld box_items %lld violations %lld\n", n.tris,
              n.pixels, n.passed, n.span_items, n.box_items, n.violations);
  return n.violations == 0 ? 0 : 1;
}
