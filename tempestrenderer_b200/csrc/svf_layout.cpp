// svf_layout.cpp - direction tables and the interpolation mesh of a direction
// layout (host side).
//
// The arithmetic that has to agree with the reference bit for bit (directions
// from (theta, phi), parabolic <-> Cartesian maps, the stratified hemisphere
// samples of the default initial guess) is written here in the reference's
// operation order and compiled without fused multiply-adds
// (-ffp-contract=off), as the reference's x86-64 build evaluates it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "svf_layout.h"

namespace svf
{

namespace
{

// SinCos_Tan (include/tempest/math/functions.hh:322-329): the reference's
// FastSinCos on the CPU.
inline void sincos_tan(float omega, float* s, float* c)
{
    float t = tanf(omega * 0.5f);
    float t2 = t * t;
    float div = 1.0f / (1.0f + t2);
    *s = 2.0f * t * div;
    *c = (1.0f - t2) * div;
}

} // namespace

void quaternion_to_euler(const float* q, float* euler)
{
    // ToMatrix3 (quaternion.hh:122-139) then Matrix3::decompose
    // (matrix3.hh:311-332); m[c][r] is column c, row r (Elements[c][r])
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float xx = x * x, xy = x * y, xz = x * z, xw = x * w, yy = y * y, yz = y * z, yw = y * w, zz = z * z,
                zw = z * w;
    const float m[3][3] = { { 1.0f - 2.0f * (yy + zz), 2.0f * (xy + zw), 2.0f * (xz - yw) },
                            { 2.0f * (xy - zw), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + xw) },
                            { 2.0f * (xz + yw), 2.0f * (yz - xw), 1.0f - 2.0f * (xx + yy) } };
    float s[3];
    for(int c = 0; c < 3; ++c)
        s[c] = sqrtf(m[c][0] * m[c][0] + m[c][1] * m[c][1] + m[c][2] * m[c][2]);
    const float pi = 3.141592f;   // MathPi (functions.hh:55)
    const float m20 = m[2][0] / s[2];
    if(m20 >= 0.9999f)
    {
        euler[0] = 0.0f;
        euler[1] = pi * 0.5f;
        euler[2] = atan2f(m[0][1], m[1][1]);
    }
    else if(m20 <= -0.9999f)
    {
        euler[0] = 0.0f;
        euler[1] = -pi * 0.5f;
        euler[2] = atan2f(m[0][1], m[1][1]);
    }
    else
    {
        euler[0] = atan2f(-m[2][1], m[2][2]);
        euler[1] = asinf(m20);
        euler[2] = atan2f(-m[1][0] / s[1], m[0][0] / s[0]);
    }
}

void angles_to_cartesian(float theta, float phi, float* w)
{
    // SphereToCartesianCoordinates (vector3.hh:375-382)
    float ct, st, cp, sp;
    sincos_tan(theta, &st, &ct);
    sincos_tan(phi, &sp, &cp);
    w[0] = cp * st;
    w[1] = sp * st;
    w[2] = ct;
}

void angles_to_parabolic(float theta, float phi, float* out)
{
    // SphereToCartesianCoordinates then CartesianToParabolicCoordinates
    // (vector3.hh:384-387), as LoadBTF derives BTF::LightsParabolic
    // (btf.cc:474-519).
    float w[3];
    angles_to_cartesian(theta, phi, w);
    out[0] = w[0] / (w[2] + 1.0f);
    out[1] = w[1] / (w[2] + 1.0f);
}

void parabolic_to_cartesian_ref(float px, float py, float* w)
{
    // vector3.hh:389-393
    float len_sq = px * px + py * py;
    w[0] = 2.0f * px / (len_sq + 1.0f);
    w[1] = 2.0f * py / (len_sq + 1.0f);
    w[2] = (1 - len_sq) / (1 + len_sq);
}

uint32_t ring81_directions(float* lp)
{
    static const int ring_deg[6] = { 0, 15, 30, 45, 60, 75 };
    static const int ring_count[6] = { 1, 6, 12, 18, 20, 24 };
    uint32_t k = 0;
    for(int r = 0; r < 6; ++r)
    {
        float theta = (float)((double)ring_deg[r] * M_PI / 180.0);
        for(int i = 0; i < ring_count[r]; ++i)
        {
            float phi = (float)(2.0 * M_PI * (double)i / (double)ring_count[r]);
            angles_to_parabolic(theta, phi, lp + 2 * k);
            ++k;
        }
    }
    return k;
}

uint32_t fibonacci_directions(uint32_t count, float* lp)
{
    // z uniform in (0, 1] on a golden-angle spiral: equal-area hemisphere lattice
    const double golden = M_PI * (3.0 - std::sqrt(5.0));
    for(uint32_t i = 0; i < count; ++i)
    {
        double z = 1.0 - (i + 0.5) / count;
        double r = std::sqrt(std::max(0.0, 1.0 - z * z));
        double phi = golden * i;
        double x = r * std::cos(phi), y = r * std::sin(phi);
        lp[2 * i] = (float)(x / (z + 1.0));
        lp[2 * i + 1] = (float)(y / (z + 1.0));
    }
    return count;
}

// ---------------------------------------------------------------------------
// Delaunay triangulation (Bowyer-Watson) of the parabolic directions
// ---------------------------------------------------------------------------

namespace
{

struct Tri
{
    int v[3];
    double cx, cy, r2;
    bool alive;
};

double orient(const double* a, const double* b, const double* c)
{
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
}

bool circumcircle(const std::vector<double>& P, Tri& t)
{
    const double* a = &P[2 * t.v[0]];
    const double* b = &P[2 * t.v[1]];
    const double* c = &P[2 * t.v[2]];
    double d = 2.0 * (a[0] * (b[1] - c[1]) + b[0] * (c[1] - a[1]) + c[0] * (a[1] - b[1]));
    if(std::fabs(d) < 1e-300)
        return false;
    double a2 = a[0] * a[0] + a[1] * a[1], b2 = b[0] * b[0] + b[1] * b[1], c2 = c[0] * c[0] + c[1] * c[1];
    t.cx = (a2 * (b[1] - c[1]) + b2 * (c[1] - a[1]) + c2 * (a[1] - b[1])) / d;
    t.cy = (a2 * (c[0] - b[0]) + b2 * (a[0] - c[0]) + c2 * (b[0] - a[0])) / d;
    t.r2 = (a[0] - t.cx) * (a[0] - t.cx) + (a[1] - t.cy) * (a[1] - t.cy);
    return true;
}

} // namespace

bool delaunay(const float* lp, uint32_t n, std::vector<uint32_t>& tris)
{
    tris.clear();
    if(n < 3)
        return false;
    std::vector<double> P(2 * (n + 3));
    double minx = 1e300, miny = 1e300, maxx = -1e300, maxy = -1e300;
    for(uint32_t i = 0; i < n; ++i)
    {
        P[2 * i] = lp[2 * i];
        P[2 * i + 1] = lp[2 * i + 1];
        minx = std::min(minx, P[2 * i]);
        maxx = std::max(maxx, P[2 * i]);
        miny = std::min(miny, P[2 * i + 1]);
        maxy = std::max(maxy, P[2 * i + 1]);
    }
    double span = std::max(maxx - minx, maxy - miny) + 1e-3;
    double mx = 0.5 * (minx + maxx), my = 0.5 * (miny + maxy);
    // super triangle
    P[2 * n] = mx - 20 * span;
    P[2 * n + 1] = my - 10 * span;
    P[2 * n + 2] = mx + 20 * span;
    P[2 * n + 3] = my - 10 * span;
    P[2 * n + 4] = mx;
    P[2 * n + 5] = my + 20 * span;
    std::vector<Tri> T;
    Tri st{ { (int)n, (int)n + 1, (int)n + 2 }, 0, 0, 0, true };
    circumcircle(P, st);
    T.push_back(st);
    const double eps = 1e-12 * span * span;
    for(uint32_t i = 0; i < n; ++i)
    {
        const double px = P[2 * i], py = P[2 * i + 1];
        std::vector<std::pair<int, int>> edges;
        for(auto& t : T)
        {
            if(!t.alive)
                continue;
            double dx = px - t.cx, dy = py - t.cy;
            if(dx * dx + dy * dy < t.r2 - eps)   // strictly inside: ties keep the triangle
            {
                t.alive = false;
                for(int e = 0; e < 3; ++e)
                    edges.emplace_back(t.v[e], t.v[(e + 1) % 3]);
            }
        }
        // boundary of the cavity: edges seen once
        std::map<std::pair<int, int>, int> cnt;
        for(auto& e : edges)
            cnt[std::make_pair(std::min(e.first, e.second), std::max(e.first, e.second))]++;
        for(auto& e : edges)
        {
            if(cnt[std::make_pair(std::min(e.first, e.second), std::max(e.first, e.second))] != 1)
                continue;
            Tri t{ { e.first, e.second, (int)i }, 0, 0, 0, true };
            if(orient(&P[2 * t.v[0]], &P[2 * t.v[1]], &P[2 * t.v[2]]) < 0)
                std::swap(t.v[0], t.v[1]);
            if(!circumcircle(P, t))
                return false;
            T.push_back(t);
        }
        // compact
        std::vector<Tri> keep;
        keep.reserve(T.size());
        for(auto& t : T)
            if(t.alive)
                keep.push_back(t);
        T.swap(keep);
    }
    for(auto& t : T)
    {
        if(t.v[0] >= (int)n || t.v[1] >= (int)n || t.v[2] >= (int)n)
            continue;
        for(int k = 0; k < 3; ++k)
            tris.push_back((uint32_t)t.v[k]);
    }
    // validation: every triangle counter-clockwise and the areas add up to the hull's
    double area = 0.0;
    for(size_t k = 0; k < tris.size(); k += 3)
    {
        double o = orient(&P[2 * tris[k]], &P[2 * tris[k + 1]], &P[2 * tris[k + 2]]);
        if(!(o > 0.0))
            return false;
        area += 0.5 * o;
    }
    // convex hull area (monotone chain)
    std::vector<uint32_t> idx(n);
    for(uint32_t i = 0; i < n; ++i)
        idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
        return P[2 * a] < P[2 * b] || (P[2 * a] == P[2 * b] && P[2 * a + 1] < P[2 * b + 1]);
    });
    std::vector<uint32_t> H(2 * n);
    int k = 0;
    for(uint32_t i = 0; i < n; ++i)
    {
        while(k >= 2 && orient(&P[2 * H[k - 2]], &P[2 * H[k - 1]], &P[2 * idx[i]]) <= 0)
            --k;
        H[k++] = idx[i];
    }
    for(int i = (int)n - 2, t = k + 1; i >= 0; --i)
    {
        while(k >= t && orient(&P[2 * H[k - 2]], &P[2 * H[k - 1]], &P[2 * idx[i]]) <= 0)
            --k;
        H[k++] = idx[i];
    }
    double hull = 0.0;
    for(int i = 0; i + 1 < k; ++i)
        hull += P[2 * H[i]] * P[2 * H[i + 1] + 1] - P[2 * H[i + 1]] * P[2 * H[i] + 1];
    hull *= 0.5;
    return std::fabs(area - hull) <= 1e-9 * std::max(1.0, std::fabs(hull));
}

uint32_t boundary_edges(const float* lp, const std::vector<uint32_t>& tris, std::vector<uint32_t>& edges,
                        std::vector<float>& angles)
{
    // LoadBTF's boundary-edge list (btf.cc:535-625): edges owned by one triangle,
    // ordered by the azimuth of their Cartesian directions.
    std::map<std::pair<uint32_t, uint32_t>, std::pair<int, uint32_t>> owner;
    for(uint32_t t = 0; t < tris.size() / 3; ++t)
        for(int e = 0; e < 3; ++e)
        {
            uint32_t a = tris[3 * t + e], b = tris[3 * t + (e + 1) % 3];
            auto key = std::make_pair(std::min(a, b), std::max(a, b));
            auto& o = owner[key];
            if(o.first == 0)
                o.second = t;
            o.first++;
        }
    struct E
    {
        uint32_t i0, i1, tri;
        float a0, a1;
    };
    std::vector<E> list;
    for(auto& kv : owner)
    {
        if(kv.second.first != 1)
            continue;
        E e{ kv.first.first, kv.first.second, kv.second.second, 0.0f, 0.0f };
        float d0[3], d1[3];
        parabolic_to_cartesian_ref(lp[2 * e.i0], lp[2 * e.i0 + 1], d0);
        parabolic_to_cartesian_ref(lp[2 * e.i1], lp[2 * e.i1 + 1], d1);
        float a0 = atan2f(d0[1], d0[0]), a1 = atan2f(d1[1], d1[0]);
        if(a0 > a1)
        {
            std::swap(e.i0, e.i1);
            std::swap(a0, a1);
        }
        if(a1 - a0 > 3.141592f)
        {
            a0 += 2.0f * 3.141592f;
            std::swap(e.i0, e.i1);
            std::swap(a0, a1);
        }
        e.a0 = a0;
        e.a1 = a1;
        list.push_back(e);
    }
    std::sort(list.begin(), list.end(), [](const E& l, const E& r) {
        if(l.a1 != r.a1)
            return l.a1 < r.a1;
        if(l.a0 != r.a0)
            return l.a0 < r.a0;
        return l.tri < r.tri;
    });
    edges.clear();
    angles.clear();
    for(auto& e : list)
    {
        edges.push_back(e.i0);
        edges.push_back(e.i1);
        edges.push_back(e.tri);
        angles.push_back(e.a0);
        angles.push_back(e.a1);
    }
    return (uint32_t)list.size();
}

// ---------------------------------------------------------------------------
// Sample tables of the default initial guess
// ---------------------------------------------------------------------------

namespace
{

constexpr float kPi = 3.141592f;   // functions.hh:55

// IntelFastRand / FloatIntelFastRand (functions.hh:214-218,249-252)
inline float lcg_float(unsigned* seed)
{
    *seed = 214013u * (*seed) + 2531011u;
    return (float)((*seed >> 16) & 0x7FFFu) / 0x7FFF;
}

// UniformSampleHemisphere (include/tempest/math/sampling3.hh:55-62)
inline void uniform_hemisphere(float ra, float rb, float* d)
{
    float r = sqrtf(1.0f - ra * ra);
    float phi = 2.0f * kPi * rb;
    float s, c;
    sincos_tan(phi, &s, &c);
    d[0] = c * r;
    d[1] = s * r;
    d[2] = ra;
}

// The stratified sample sequence of StratifiedMonteCarloIntegratorHemisphere
// (numerical-methods.hh:210-237) and, run by one worker in index order,
// ParallelStratifiedMonteCarloIntegratorHemisphere (:261-304) and the PCA search
// (svbrdf-fitting-pipeline.cc:450-469): seed 1, x then y jitter per sample.
void stratified_hemisphere(uint32_t samples, std::vector<float>& dirs)
{
    unsigned seed = 1;
    float sq = sqrtf((float)samples);
    uint32_t sqi = (uint32_t)(int32_t)sq;
    dirs.resize(3 * (size_t)samples);
    for(uint32_t i = 0; i < samples; ++i)
    {
        uint32_t xi = i % sqi, yi = i / sqi;
        float x = (xi + lcg_float(&seed)) / sq;
        float y = (yi + lcg_float(&seed)) / sq;
        uniform_hemisphere(x, y, &dirs[3 * (size_t)i]);
    }
}

// CartesianToParabolicMapCoordinates (vector3.hh:400-403) and the bilinear
// set-up of Texture::sample (texture.hh:495-516) on the 64x64 NDF map, with
// FastFloorToInt64 (functions.hh:82-88) and Modulo (:547-550).
inline void bilinear_setup(const float* d, int32_t* cell, float* fx1, float* fy1)
{
    float tx = d[0] / (d[2] + 1.0f) * 0.5f + 0.5f;
    float ty = d[1] / (d[2] + 1.0f) * 0.5f + 0.5f;
    const int64_t W = 64;
    float ux = W * tx - 0.5f, uy = W * ty - 0.5f;
    int64_t xt = (int64_t)ux - (std::signbit(ux) ? 1 : 0);
    int64_t yt = (int64_t)uy - (std::signbit(uy) ? 1 : 0);
    int64_t x0 = ((xt % W) + W) % W, y0 = ((yt % W) + W) % W;
    *cell = (int32_t)(x0 + W * y0);
    *fx1 = ux - (float)xt;
    *fy1 = uy - (float)yt;
}

} // namespace

void build_init_host_tables(InitHostTables& t)
{
    const float pdf = 1.0f / (2.0f * kPi);
    t.pdf = pdf;

    // NDF integrand samples (4096) and the NDF texels inside the hemisphere
    stratified_hemisphere(4096, t.ndf_dirs);
    t.ndf_row_texel.clear();
    t.ndf_row_normal.clear();
    for(uint32_t y = 0; y < 64; ++y)
        for(uint32_t x = 0; x < 64; ++x)
        {
            // NDFRecord (svbrdf-fitting-pipeline.cc:118-125):
            // ParabolicMapToCartesianCoordinates of (x/63, y/63)
            float tx = (float)x / (64 - 1), ty = (float)y / (64 - 1);
            float n[3];
            parabolic_to_cartesian_ref(2.0f * tx - 1.0f, 2.0f * ty - 1.0f, n);
            if(n[2] <= 0.0f)
                continue;
            t.ndf_row_texel.push_back((int32_t)(y * 64 + x));
            t.ndf_row_normal.insert(t.ndf_row_normal.end(), n, n + 3);
        }
    t.ndf_scale = 1.0 / (double)((float)4096 * pdf);

    // ndf_denom: 256x256 samples of the bilinear NDF (pipeline.cc:403-406), a fixed
    // linear functional of the NDF texels
    {
        std::vector<float> dirs;
        stratified_hemisphere(65536, dirs);
        std::vector<double> w(4096, 0.0);
        const double scale = 1.0 / (double)((float)65536 * pdf);
        for(uint32_t s = 0; s < 65536; ++s)
        {
            int32_t cell;
            float fx1, fy1;
            bilinear_setup(&dirs[3 * s], &cell, &fx1, &fy1);
            int x0 = cell % 64, y0 = cell / 64, x1 = (x0 + 1) % 64, y1 = (y0 + 1) % 64;
            float fx0 = 1.0f - fx1, fy0 = 1.0f - fy1;
            w[y0 * 64 + x0] += (double)fx0 * fy0 * scale;
            w[y0 * 64 + x1] += (double)fx1 * fy0 * scale;
            w[y1 * 64 + x0] += (double)fx0 * fy1 * scale;
            w[y1 * 64 + x1] += (double)fx1 * fy1 * scale;
        }
        t.denom_w.assign(w.begin(), w.end());
    }

    // PCA search: 512x512 samples, grouped by bilinear cell (stable in sample order)
    {
        std::vector<float> dirs;
        stratified_hemisphere(512 * 512, dirs);
        const uint32_t S = 512 * 512;
        std::vector<int32_t> cell(S);
        std::vector<float> fx(S), fy(S);
        for(uint32_t s = 0; s < S; ++s)
            bilinear_setup(&dirs[3 * s], &cell[s], &fx[s], &fy[s]);
        std::vector<uint32_t> order(S);
        for(uint32_t s = 0; s < S; ++s)
            order[s] = s;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cell[a] < cell[b]; });
        t.pca_index.resize(S);
        t.pca_frac.resize(2 * (size_t)S);
        t.pca_cell_id.clear();
        t.pca_cell_start.clear();
        for(uint32_t k = 0; k < S; ++k)
        {
            uint32_t s = order[k];
            if(k == 0 || cell[s] != cell[order[k - 1]])
            {
                t.pca_cell_id.push_back(cell[s]);
                t.pca_cell_start.push_back(k);
            }
            t.pca_index[k] = s;
            t.pca_frac[2 * k] = fx[s];
            t.pca_frac[2 * k + 1] = fy[s];
        }
        t.pca_cell_start.push_back(S);
        t.pca_dir.resize(4 * (size_t)S);
        for(uint32_t s = 0; s < S; ++s)
        {
            t.pca_dir[4 * s] = dirs[3 * s];
            t.pca_dir[4 * s + 1] = dirs[3 * s + 1];
            t.pca_dir[4 * s + 2] = dirs[3 * s + 2];
            t.pca_dir[4 * s + 3] = 0.0f;
        }
    }

    // SGGX projection samples (pipeline.cc:639, 1024 samples)
    {
        std::vector<float> dirs;
        stratified_hemisphere(1024, dirs);
        t.proj_dir.resize(4 * 1024);
        t.proj_frac.resize(2 * 1024);
        t.proj_cell.resize(1024);
        for(uint32_t s = 0; s < 1024; ++s)
        {
            t.proj_dir[4 * s] = dirs[3 * s];
            t.proj_dir[4 * s + 1] = dirs[3 * s + 1];
            t.proj_dir[4 * s + 2] = dirs[3 * s + 2];
            t.proj_dir[4 * s + 3] = 0.0f;
            bilinear_setup(&dirs[3 * s], &t.proj_cell[s], &t.proj_frac[2 * s], &t.proj_frac[2 * s + 1]);
        }
    }

    // Matrix2::rotation(2 pi / (512 - 1)) (matrix2.hh:66-73, pipeline.cc:608)
    sincos_tan(2.0f * kPi / (512 - 1), &t.rot_s, &t.rot_c);
    // PCA fill value: the NDF at (0, 0, 1) (pipeline.cc:444-445)
    {
        float up[3] = { 0.0f, 0.0f, 1.0f };
        bilinear_setup(up, &t.axis_cell, &t.axis_frac[0], &t.axis_frac[1]);
    }
}

// MurmurHash3's 32-bit finaliser (fmix32), the reference's Hash32
// (functions.hh:220-229).
static uint32_t fmix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

bool downsample_light_view(uint32_t L, uint32_t n, uint32_t* idx)
{
    // DownsampleLightView (svbrdf-lsq-fitting-setup.cc:129-163): direction k of
    // n is drawn in [ceil(r k), ceil(r (k + 1))), r = (L - 1) / (n - 1), by
    // FastRandRange (min + Hash32(seed) % (max - min), seed 42 carried along),
    // redrawn while it repeats the previous draw
    if(n < 2 || n >= L)
        return false;
    const float step = (float)(L - 1) / (float)(n - 1);
    uint32_t last = ~0u, lo = 0, seed = 42;
    for(uint32_t k = 0; k < n; ++k)
    {
        const uint32_t c = (uint32_t)std::ceil(step * (float)(k + 1));
        const uint32_t hi = c < L ? c : L;
        if(hi <= lo)
            return false;
        uint32_t s;
        uint32_t guard = 0;
        do
        {
            seed = fmix32(seed);
            s = lo + seed % (hi - lo);
            if(++guard > 1000000u)
                return false;   // (one value in range and it repeats the last: the reference would not end)
        } while(s == last);
        last = s;
        idx[k] = s;
        lo = hi;
    }
    return true;
}

} // namespace svf
