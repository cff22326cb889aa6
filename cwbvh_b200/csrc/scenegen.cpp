// Seeded procedural scenes.  The reference measures on its own mesh.dat, which
// is not shipped; these generators produce the synthetic scenes of the
// benchmark configurations instead.  Every random quantity is
// hash(seed, stream, index), so a scene depends only on its parameters.
#include <algorithm>
#include <cmath>

#include "host_common.h"

namespace rq {
namespace {

int32_t add_vertex(Mesh& m, V3 p) {
    m.v.push_back(p.x);
    m.v.push_back(p.y);
    m.v.push_back(p.z);
    return (int32_t)(m.v.size() / 3 - 1);
}
void add_tri(Mesh& m, int32_t a, int32_t b, int32_t c) {
    m.i.push_back(a);
    m.i.push_back(b);
    m.i.push_back(c);
}
void add_quad(Mesh& m, int32_t a, int32_t b, int32_t c, int32_t d) {
    add_tri(m, a, b, c);
    add_tri(m, a, c, d);
}

// Axis-aligned box, 12 triangles wound counter-clockwise seen from outside.
void add_box(Mesh& m, V3 lo, V3 hi) {
    int32_t k[8];
    for (int c = 0; c < 8; ++c)
        k[c] = add_vertex(m, v3((c & 1) ? hi.x : lo.x, (c & 2) ? hi.y : lo.y, (c & 4) ? hi.z : lo.z));
    add_quad(m, k[0], k[4], k[6], k[2]);  // -x
    add_quad(m, k[1], k[3], k[7], k[5]);  // +x
    add_quad(m, k[0], k[1], k[5], k[4]);  // -y
    add_quad(m, k[2], k[6], k[7], k[3]);  // +y
    add_quad(m, k[0], k[2], k[3], k[1]);  // -z
    add_quad(m, k[4], k[5], k[7], k[6]);  // +z
}

// Regular grid of (nx+1) x (ny+1) vertices, heights from f(i, j); upward winding.
template <typename F>
void add_grid(Mesh& m, int nx, int ny, float x0, float y0, float sx, float sy, F height) {
    const int32_t base = (int32_t)(m.v.size() / 3);
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) add_vertex(m, v3(x0 + sx * i, y0 + sy * j, height(i, j)));
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int32_t v00 = base + j * (nx + 1) + i, v10 = v00 + 1;
            const int32_t v01 = v00 + (nx + 1), v11 = v01 + 1;
            add_tri(m, v00, v10, v11);
            add_tri(m, v00, v11, v01);
        }
}

}  // namespace

// (grid+1)^2-vertex heightfield over [0,1]^2 with heights U[0,1] (2*grid^2
// triangles) plus n_boxes boxes with centres U[0,1]^3 and edges U[bmin,bmax].
void gen_heightfield_boxes(uint64_t seed, int grid, int n_boxes, float bmin, float bmax, Mesh& m) {
    m = Mesh();
    m.v.reserve(3 * ((size_t)(grid + 1) * (grid + 1) + 8 * (size_t)n_boxes));
    m.i.reserve(3 * (2 * (size_t)grid * grid + 12 * (size_t)n_boxes));
    const float s = 1.0f / (float)grid;
    add_grid(m, grid, grid, 0.f, 0.f, s, s,
             [&](int i, int j) { return u01(seed, 1, (uint64_t)j * (grid + 1) + i); });
    for (int b = 0; b < n_boxes; ++b) {
        const V3 c = v3(u01(seed, 2, b), u01(seed, 3, b), u01(seed, 4, b));
        const V3 e = v3(bmin + (bmax - bmin) * u01(seed, 5, b), bmin + (bmax - bmin) * u01(seed, 6, b),
                        bmin + (bmax - bmin) * u01(seed, 7, b));
        add_box(m, c - e * 0.5f, c + e * 0.5f);
    }
}

// City: n_buildings on a square lot grid (lot 20 x 20 units) over a ground
// grid.  Buildings are instances of a few templates -- boxes and hexagonal
// prisms whose walls are split into floors and columns -- scaled, rotated and
// flattened into one mesh.  Heights are log-normal (median 24, sigma 0.6,
// clamped to [6, 200]); about 100 triangles per building.
void gen_city(uint64_t seed, int n_buildings, Mesh& m) {
    m = Mesh();
    const int side = (int)std::ceil(std::sqrt((double)std::max(1, n_buildings)));
    const float lot = 20.0f, extent = lot * side;
    const int ground = std::min(512, side * 2);
    add_grid(m, ground, ground, 0.f, 0.f, extent / ground, extent / ground, [](int, int) { return 0.0f; });
    const float kPi = 3.14159265358979f;
    for (int b = 0; b < n_buildings; ++b) {
        const int gx = b % side, gy = b / side;
        const float cx = (gx + 0.5f) * lot, cy = (gy + 0.5f) * lot;
        const float w = 8.0f + 8.0f * u01(seed, 11, b), d = 8.0f + 8.0f * u01(seed, 12, b);
        // Box-Muller normal for the log-normal height.
        const float u1 = std::max(1e-7f, u01(seed, 13, b)), u2 = u01(seed, 14, b);
        const float g = std::sqrt(-2.0f * std::log(u1)) * std::cos(2.0f * kPi * u2);
        const float h = std::min(200.0f, std::max(6.0f, 24.0f * std::exp(0.6f * g)));
        const float rot = 2.0f * kPi * u01(seed, 15, b);
        const float cr = std::cos(rot), sr = std::sin(rot);
        const bool prism = u01(seed, 16, b) < 0.35f;
        const int floors = std::max(1, std::min(8, (int)std::lround(h / 8.0f)));
        const int sides = prism ? 6 : 4;
        const int cols = prism ? 2 : 3;
        // Footprint ring of the template, then the instance transform.
        std::vector<V3> ring;
        for (int k = 0; k < sides; ++k) {
            float x, y;
            if (prism) {
                const float a = 2.0f * kPi * k / sides;
                x = 0.5f * std::cos(a);
                y = 0.5f * std::sin(a);
            } else {
                const float cxk[4] = {-0.5f, 0.5f, 0.5f, -0.5f}, cyk[4] = {-0.5f, -0.5f, 0.5f, 0.5f};
                x = cxk[k];
                y = cyk[k];
            }
            x *= w;
            y *= d;
            ring.push_back(v3(cx + cr * x - sr * y, cy + sr * x + cr * y, 0.f));
        }
        for (int k = 0; k < sides; ++k) {
            const V3 a = ring[k], bb = ring[(k + 1) % sides];
            const int32_t base = (int32_t)(m.v.size() / 3);
            for (int f = 0; f <= floors; ++f)
                for (int c = 0; c <= cols; ++c) {
                    const float t = (float)c / cols;
                    V3 p = a + (bb - a) * t;
                    p.z = h * f / floors;
                    add_vertex(m, p);
                }
            for (int f = 0; f < floors; ++f)
                for (int c = 0; c < cols; ++c) {
                    const int32_t v00 = base + f * (cols + 1) + c, v10 = v00 + 1;
                    const int32_t v01 = v00 + (cols + 1), v11 = v01 + 1;
                    add_quad(m, v00, v10, v11, v01);
                }
        }
        const int32_t roof = (int32_t)(m.v.size() / 3);
        for (int k = 0; k < sides; ++k) add_vertex(m, v3(ring[k].x, ring[k].y, h));
        for (int k = 1; k + 1 < sides; ++k) add_tri(m, roof, roof + k, roof + k + 1);
    }
}

// Large scene: displaced terrain tiles (half the triangles) plus displaced
// tessellated spheres (the other half), sized to about target_tris.
void gen_spheres_terrain(uint64_t seed, int64_t target_tris, Mesh& m) {
    m = Mesh();
    const float kPi = 3.14159265358979f;
    const int64_t terrain_tris = target_tris / 2;
    const int tiles_side = (int)std::max<int64_t>(1, (int64_t)std::sqrt((double)terrain_tris / (2.0 * 256 * 256)));
    const int tile_res = (int)std::max<int64_t>(
        2, (int64_t)std::sqrt((double)terrain_tris / (2.0 * tiles_side * tiles_side)));
    const float tile = 100.0f;
    float ph[8];
    for (int k = 0; k < 8; ++k) ph[k] = 2.0f * kPi * u01(seed, 21, k);
    auto terrain_h = [&](float x, float y) {
        return 6.0f * std::sin(0.031f * x + ph[0]) * std::cos(0.027f * y + ph[1]) +
               2.5f * std::sin(0.11f * x + ph[2]) * std::sin(0.093f * y + ph[3]) +
               0.8f * std::sin(0.41f * x + ph[4]) * std::cos(0.37f * y + ph[5]);
    };
    for (int ty = 0; ty < tiles_side; ++ty)
        for (int tx = 0; tx < tiles_side; ++tx) {
            const float x0 = tx * tile, y0 = ty * tile, s = tile / tile_res;
            add_grid(m, tile_res, tile_res, x0, y0, s, s,
                     [&](int i, int j) { return terrain_h(x0 + s * i, y0 + s * j); });
        }
    const int64_t sphere_tris = target_tris - m.nt();
    const int n_spheres = (int)std::max<int64_t>(1, sphere_tris / 20000);
    const int64_t per = std::max<int64_t>(8, sphere_tris / n_spheres);
    const int segs = (int)std::max<int64_t>(4, (int64_t)std::sqrt((double)per));
    const int rings = (int)std::max<int64_t>(2, per / (2 * segs));
    const float world = tiles_side * tile;
    for (int k = 0; k < n_spheres; ++k) {
        const float r = 2.0f + 6.0f * u01(seed, 22, k);
        const float cx = world * u01(seed, 23, k), cy = world * u01(seed, 24, k);
        const V3 c = v3(cx, cy, terrain_h(cx, cy) + r * (0.6f + 1.5f * u01(seed, 25, k)));
        const float f1 = 3.0f + 5.0f * u01(seed, 26, k), f2 = 2.0f + 4.0f * u01(seed, 27, k);
        const int32_t base = (int32_t)(m.v.size() / 3);
        for (int i = 0; i <= rings; ++i) {
            const float th = kPi * i / rings;
            for (int j = 0; j <= segs; ++j) {
                const float phv = 2.0f * kPi * j / segs;
                const float disp = 1.0f + 0.08f * std::sin(f1 * th) * std::cos(f2 * phv);
                const float rr = r * disp;
                add_vertex(m, v3(c.x + rr * std::sin(th) * std::cos(phv), c.y + rr * std::sin(th) * std::sin(phv),
                                 c.z + rr * std::cos(th)));
            }
        }
        for (int i = 0; i < rings; ++i)
            for (int j = 0; j < segs; ++j) {
                const int32_t v00 = base + i * (segs + 1) + j, v10 = v00 + 1;
                const int32_t v01 = v00 + (segs + 1), v11 = v01 + 1;
                if (i != 0) add_tri(m, v00, v11, v10);
                if (i != rings - 1) add_tri(m, v00, v01, v11);
            }
    }
}

}  // namespace rq
