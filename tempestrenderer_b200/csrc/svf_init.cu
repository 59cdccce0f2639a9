// svf_init.cu - the reference's default initial guess on the GPU
// (SVBRDFFitPipeline::fit, tools/svbrdf-fitting/svbrdf-fitting-pipeline.cc:350-660).
//
//   1. NDF texture: NDF(n_j) = 2pi/4096 sum_s lum(l_s, reflect(l_s, n_j)) with
//      barycentric interpolation of the luminance slice on the direction mesh
//      (NDFRecord :110-133, BTFSampleLuminanceSlice btf.hh:229-257).  The sample
//      directions are the same for every texel, so the NDF is a fixed linear map
//      of the slice: NDF = Op * lum.  Op ([rows][N], rows = NDF texels inside the
//      hemisphere) is built once per direction layout (ndf_operator_kernel) and
//      applied to all texels as one tensor-core GEMM (svf_ndf_tc.cu).
//   2. Per texel (init_finish_kernel): ndf_denom (a fixed linear functional of the
//      NDF), the PCA normal search (argmax of the bilinear NDF over 512^2
//      directions, pruned per bilinear cell), the tangent search (512 in-plane
//      rotations), the SGGX projection integral and Matrix3::decompose.
//
// Arithmetic that decides which sample wins an argmax (bilinear lookups, the
// tangent recurrence, point location in the mesh) uses round-to-nearest
// intrinsics, never fused multiply-adds, so that it reproduces the reference's
// float results.
#include <cuda_runtime.h>
#include <stdint.h>

#include "svf_internal.h"

namespace svf
{

namespace
{

constexpr float kPi = 3.141592f;   // functions.hh:55

__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dvd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float dot3(const float* a, const float* b)
{
    return add(add(mul(a[0], b[0]), mul(a[1], b[1])), mul(a[2], b[2]));
}

// ---------------------------------------------------------------------------
// point location on the direction mesh
// ---------------------------------------------------------------------------

// TriangleBarycentricCoordinates (include/tempest/math/intersect.hh:383-401)
__device__ __forceinline__ void tri_bary(float px, float py, const float* v0, const float* v1, const float* v2, float* bx,
                                         float* by)
{
    float x1_x3 = sub(v1[0], v0[0]), x2_x3 = sub(v2[0], v0[0]), x_x3 = sub(px, v0[0]);
    float y1_y3 = sub(v1[1], v0[1]), y2_y3 = sub(v2[1], v0[1]), y_y3 = sub(py, v0[1]);
    float det = sub(mul(x1_x3, y2_y3), mul(x2_x3, y1_y3));
    if(det < 1e-9f)
    {
        float dx = sub(px, v0[0]), dy = sub(py, v0[1]);
        *bx = *by = __fsqrt_rn(add(mul(dx, dx), mul(dy, dy)));
        return;
    }
    *bx = dvd(sub(mul(y2_y3, x_x3), mul(x2_x3, y_y3)), det);
    *by = dvd(add(mul(-y1_y3, x_x3), mul(x1_x3, y_y3)), det);
}

// The first triangle, in index order, whose IntersectTriangle test passes
// (intersect.hh:403-419); outside the mesh, IntersectEdge (btf.hh:271-321).
// The reference walks a BVH instead of the index order; the two can differ
// only for a point on an edge shared by two triangles, where both give the
// same interpolant.
__device__ void locate(const float* lp, const uint32_t* tri, uint32_t ntri, const uint32_t* edges, const float* eang,
                       uint32_t nedge, const float* d, uint32_t* out_tri, float* bary)
{
    float zp1 = add(d[2], 1.0f);
    float px = dvd(d[0], zp1), py = dvd(d[1], zp1);
    for(uint32_t t = 0; t < ntri; ++t)
    {
        const uint32_t* v = tri + 3 * t;
        float bx, by;
        tri_bary(px, py, lp + 2 * v[0], lp + 2 * v[1], lp + 2 * v[2], &bx, &by);
        float w = sub(sub(1.0f, bx), by);
        if(0.0f > bx || bx > 1.0f || 0.0f > by || by > 1.0f || 0.0f > w || w > 1.0f)
            continue;
        *out_tri = t;
        bary[0] = bx;
        bary[1] = by;
        bary[2] = w;
        return;
    }
    float angle = atan2f(d[1], d[0]);
    uint32_t first = 0, count = nedge;
    while(count > 0)
    {
        uint32_t step = count / 2, it = first + step;
        if(eang[2 * it + 1] < angle)
        {
            first = it + 1;
            count -= step + 1;
        }
        else
            count = step;
    }
    if(first == nedge)
        first = 0;
    const uint32_t* e = edges + 3 * first;
    const uint32_t t = e[2];
    const uint32_t* v = tri + 3 * t;
    float ratio = dvd(sub(angle, eang[2 * first]), sub(eang[2 * first + 1], eang[2 * first]));
    float om = sub(1.0f, ratio);
    float qx = add(mul(om, lp[2 * e[0]]), mul(ratio, lp[2 * e[1]]));
    float qy = add(mul(om, lp[2 * e[0] + 1]), mul(ratio, lp[2 * e[1] + 1]));
    float bx, by;
    tri_bary(qx, qy, lp + 2 * v[0], lp + 2 * v[1], lp + 2 * v[2], &bx, &by);
    bx = fminf(fmaxf(bx, 0.0f), 1.0f);
    by = fminf(fmaxf(by, 0.0f), 1.0f);
    *out_tri = t;
    bary[0] = bx;
    bary[1] = by;
    bary[2] = sub(sub(1.0f, bx), by);
}

// Loads the mesh into shared memory: lp [2L], tri [3T], edges [3E], eang [2E].
struct MeshSmem
{
    float* lp;
    uint32_t* tri;
    uint32_t* edges;
    float* eang;
};

__device__ __forceinline__ MeshSmem load_mesh(const MeshDevice& m, uint32_t L, unsigned char* base)
{
    MeshSmem s;
    s.lp = reinterpret_cast<float*>(base);
    s.tri = reinterpret_cast<uint32_t*>(s.lp + 2 * L);
    s.edges = s.tri + 3 * m.ntri;
    s.eang = reinterpret_cast<float*>(s.edges + 3 * m.nedge);
    for(uint32_t i = threadIdx.x; i < 2 * L; i += blockDim.x)
        s.lp[i] = m.lp[i];
    for(uint32_t i = threadIdx.x; i < 3 * m.ntri; i += blockDim.x)
        s.tri[i] = m.tri[i];
    for(uint32_t i = threadIdx.x; i < 3 * m.nedge; i += blockDim.x)
        s.edges[i] = m.edges[i];
    for(uint32_t i = threadIdx.x; i < 2 * m.nedge; i += blockDim.x)
        s.eang[i] = m.eang[i];
    return s;
}

__host__ __device__ inline size_t mesh_smem_bytes(uint32_t L, uint32_t ntri, uint32_t nedge)
{
    size_t b = sizeof(float) * 2 * L + sizeof(uint32_t) * 3 * (ntri + nedge) + sizeof(float) * 2 * nedge;
    return (b + 15) & ~size_t(15);
}

// Locates the 4096 light directions of the NDF integrand once.
__global__ void locate_lights_kernel(MeshDevice mesh, uint32_t L, const float* __restrict__ dirs, int32_t* light_tri,
                                     float* light_bary)
{
    extern __shared__ __align__(16) unsigned char smem[];
    MeshSmem m = load_mesh(mesh, L, smem);
    __syncthreads();
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= (uint32_t)kNdfSamples)
        return;
    const float* d = dirs + 3 * s;
    if(d[2] < 0.0f)
    {
        light_tri[s] = -1;
        return;
    }
    uint32_t t;
    float b[3];
    locate(m.lp, m.tri, mesh.ntri, m.edges, m.eang, mesh.nedge, d, &t, b);
    light_tri[s] = (int32_t)t;
    light_bary[3 * s] = b[0];
    light_bary[3 * s + 1] = b[1];
    light_bary[3 * s + 2] = b[2];
}

// One CTA per operator row: accumulates the 9 interpolation weights of every
// (light sample, reflected view) pair in FP64 shared memory, then writes the row
// scaled by 1/(4096 pdf).
__global__ void __launch_bounds__(256) ndf_operator_kernel(MeshDevice mesh, uint32_t L, uint32_t N, uint32_t k_pad,
                                                           const float* __restrict__ dirs,
                                                           const float* __restrict__ normals,
                                                           const int32_t* __restrict__ light_tri,
                                                           const float* __restrict__ light_bary, double scale,
                                                           float* __restrict__ op)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double* acc = reinterpret_cast<double*>(smem);
    MeshSmem m = load_mesh(mesh, L, smem + sizeof(double) * N);
    for(uint32_t k = threadIdx.x; k < N; k += blockDim.x)
        acc[k] = 0.0;
    const float* n = normals + 3 * blockIdx.x;
    const float nrm[3] = { n[0], n[1], n[2] };
    __syncthreads();
    for(uint32_t s = threadIdx.x; s < (uint32_t)kNdfSamples; s += blockDim.x)
    {
        const int32_t lt = light_tri[s];
        if(lt < 0)
            continue;
        const float* l = dirs + 3 * s;
        // Reflect (vector3.hh:420): 2 (n . l) n - l
        float d2 = mul(2.0f, dot3(nrm, l));
        float v[3] = { sub(mul(d2, nrm[0]), l[0]), sub(mul(d2, nrm[1]), l[1]), sub(mul(d2, nrm[2]), l[2]) };
        if(v[2] < 0.0f)
            continue;
        uint32_t vt;
        float vb[3];
        locate(m.lp, m.tri, mesh.ntri, m.edges, m.eang, mesh.nedge, v, &vt, vb);
        const float* lb = light_bary + 3 * s;
        for(int vi = 0; vi < 3; ++vi)
        {
            const uint32_t vv = m.tri[3 * vt + vi];
            const float wv = vb[(vi + 2) % 3];
            for(int li = 0; li < 3; ++li)
            {
                const uint32_t lv = m.tri[3 * lt + li];
                const float wl = lb[(li + 2) % 3];
                atomicAdd(&acc[vv * L + lv], (double)mul(wl, wv));
            }
        }
    }
    __syncthreads();
    float* row = op + (uint64_t)blockIdx.x * k_pad;
    for(uint32_t k = threadIdx.x; k < k_pad; k += blockDim.x)
        row[k] = k < N ? (float)(acc[k] * scale) : 0.0f;
}

// ---------------------------------------------------------------------------
// per-texel finish of the initial guess
// ---------------------------------------------------------------------------

// Texture::sample bilinear combination (texture.hh:508-519) for cell x0 + 64 y0
// with fractions (fx1, fy1), wrapping.
__device__ __forceinline__ float bilinear(const float* ndf, int32_t cell, float fx1, float fy1)
{
    int x0 = cell & 63, y0 = cell >> 6;
    int x1 = (x0 + 1) & 63, y1 = (y0 + 1) & 63;
    float c00 = ndf[y0 * 64 + x0], c01 = ndf[y0 * 64 + x1], c10 = ndf[y1 * 64 + x0], c11 = ndf[y1 * 64 + x1];
    float fx0 = sub(1.0f, fx1), fy0 = sub(1.0f, fy1);
    return add(mul(add(mul(fx0, c00), mul(fx1, c01)), fy0), mul(add(mul(fx0, c10), mul(fx1, c11)), fy1));
}

__device__ __forceinline__ float cell_bound(const float* ndf, int32_t cell)
{
    int x0 = cell & 63, y0 = cell >> 6;
    int x1 = (x0 + 1) & 63, y1 = (y0 + 1) & 63;
    return fmaxf(fmaxf(ndf[y0 * 64 + x0], ndf[y0 * 64 + x1]), fmaxf(ndf[y1 * 64 + x0], ndf[y1 * 64 + x1]));
}

// CartesianToParabolicMapCoordinates + bilinear set-up (texture.hh:495-516).
__device__ __forceinline__ float ndf_at(const float* ndf, const float* d)
{
    float zp1 = add(d[2], 1.0f);
    float tx = add(mul(dvd(d[0], zp1), 0.5f), 0.5f);
    float ty = add(mul(dvd(d[1], zp1), 0.5f), 0.5f);
    float ux = sub(mul(64.0f, tx), 0.5f), uy = sub(mul(64.0f, ty), 0.5f);
    long long xt = (long long)ux - (signbit(ux) ? 1 : 0);
    long long yt = (long long)uy - (signbit(uy) ? 1 : 0);
    int x0 = (int)(((xt % 64) + 64) % 64), y0 = (int)(((yt % 64) + 64) % 64);
    return bilinear(ndf, x0 + 64 * y0, sub(ux, (float)xt), sub(uy, (float)yt));
}

// PCAIntegrand (pipeline.cc:161-173)
__device__ __forceinline__ float pca_value(const float* ndf, const float* d)
{
    return d[2] < 0.0f ? 0.0f : ndf_at(ndf, d);
}

// argmax with the reference's tie rule: larger value, then lower sample index
__device__ __forceinline__ bool better(float v, uint32_t i, float bv, uint32_t bi)
{
    return v > bv || (v == bv && i < bi);
}

__device__ __forceinline__ void warp_argmax(float& v, uint32_t& i)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
    {
        float ov = __shfl_xor_sync(0xffffffffu, v, o);
        uint32_t oi = __shfl_xor_sync(0xffffffffu, i, o);
        if(better(ov, oi, v, i))
        {
            v = ov;
            i = oi;
        }
    }
}

constexpr int kFinishThreads = 256;

__device__ void block_argmax(float& v, uint32_t& i, float* sv, uint32_t* si)
{
    warp_argmax(v, i);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if(lane == 0)
    {
        sv[warp] = v;
        si[warp] = i;
    }
    __syncthreads();
    if(warp == 0)
    {
        v = lane < kFinishThreads / 32 ? sv[lane] : -INFINITY;
        i = lane < kFinishThreads / 32 ? si[lane] : 0xffffffffu;
        warp_argmax(v, i);
        if(lane == 0)
        {
            sv[0] = v;
            si[0] = i;
        }
    }
    __syncthreads();
    v = sv[0];
    i = si[0];
    __syncthreads();
}

__device__ double block_sum(double x, double* sd)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if(lane == 0)
        sd[warp] = x;
    __syncthreads();
    double s = 0.0;
    for(int w = 0; w < kFinishThreads / 32; ++w)
        s += sd[w];
    __syncthreads();
    return s;
}

__global__ void __launch_bounds__(kFinishThreads) init_finish_kernel(InitLayout lay, const float* __restrict__ ndf_rows,
                                                                     uint32_t ldr, float* __restrict__ init,
                                                                     float* __restrict__ info,
                                                                     float* __restrict__ ndf_out)
{
    __shared__ __align__(16) float ndf[kNdfTexels];
    __shared__ float tan_seq[3][kTangentSteps];
    __shared__ float sv[32];
    __shared__ uint32_t si[32];
    __shared__ double sd[32];
    __shared__ float sh_n[3], sh_B[9];
    const uint64_t t = blockIdx.x;
    // the operator rows are the NDF texels inside the hemisphere; the rest are 0
    // (NDFRecord, pipeline.cc:118-123)
    for(uint32_t i = threadIdx.x; i < kNdfTexels; i += kFinishThreads)
        ndf[i] = 0.0f;
    __syncthreads();
    const float* src = ndf_rows + t * ldr;
    for(uint32_t r = threadIdx.x; r < lay.ndf_rows; r += kFinishThreads)
        ndf[lay.ndf_row_texel[r]] = src[r];
    __syncthreads();
    if(ndf_out)
        for(uint32_t i = threadIdx.x; i < kNdfTexels; i += kFinishThreads)
            ndf_out[t * kNdfTexels + i] = ndf[i];

    // ndf_denom (pipeline.cc:403-406)
    double part = 0.0;
    for(uint32_t j = threadIdx.x; j < kNdfTexels; j += kFinishThreads)
        part += (double)lay.denom_w[j] * (double)ndf[j];
    const float ndf_denom = (float)block_sum(part, sd);
    const float ndf_norm = 1 / ndf_denom;

    // PCA normal search (pipeline.cc:429-489)
    const float v0 = bilinear(ndf, lay.axis_cell, lay.axis_fx1, lay.axis_fy1);
    float bv = -INFINITY;
    uint32_t bc = 0xffffffffu;
    for(uint32_t c = threadIdx.x; c < lay.pca_cells; c += kFinishThreads)
    {
        float u = cell_bound(ndf, lay.pca_cell_id[c]);
        if(better(u, c, bv, bc))
        {
            bv = u;
            bc = c;
        }
    }
    block_argmax(bv, bc, sv, si);
    // a texel whose NDF holds NaN has no ordered cell: search cell 0 (its fit is
    // flagged non-finite later)
    if(bc >= lay.pca_cells)
        bc = 0;
    // best sample of the most promising cell gives the pruning bound
    float B = -INFINITY;
    {
        const uint32_t s0 = lay.pca_cell_start[bc], s1 = lay.pca_cell_start[bc + 1];
        const int32_t cell = lay.pca_cell_id[bc];
        float mv = -INFINITY;
        uint32_t mi = 0xffffffffu;
        for(uint32_t k = s0 + threadIdx.x; k < s1; k += kFinishThreads)
        {
            float2 fr = lay.pca_frac[k];
            float v = bilinear(ndf, cell, fr.x, fr.y);
            if(better(v, lay.pca_index[k], mv, mi))
            {
                mv = v;
                mi = lay.pca_index[k];
            }
        }
        block_argmax(mv, mi, sv, si);
        B = mv;
    }
    // every sample that can reach B lives in a cell whose corner maximum reaches
    // it (bilinear weights are in [0, 1]; the slack covers their rounding)
    // A warp per cell, its lanes over the cell's samples (a cell holds about 64):
    // the work of the cells that pass is spread over all threads whichever cells
    // they are.  Each warp tests 32 cells at a time, one per lane, and walks the
    // passing ones (the argmax's tie rule makes the order irrelevant).
    float best_v = -INFINITY;
    uint32_t best_i = 0xffffffffu;
    {
        const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
        for(uint32_t c0 = warp * 32u; c0 < lay.pca_cells; c0 += kFinishThreads)
        {
            const uint32_t c = c0 + lane;
            bool pass = false;
            if(c < lay.pca_cells)
            {
                const float u = cell_bound(ndf, lay.pca_cell_id[c]);
                pass = !(u + fabsf(u) * 1e-5f < B);
            }
            for(uint32_t m = __ballot_sync(0xffffffffu, pass); m; m &= m - 1)
            {
                const uint32_t cc = c0 + (uint32_t)(__ffs(m) - 1);
                const int32_t cell = lay.pca_cell_id[cc];
                for(uint32_t k = lay.pca_cell_start[cc] + lane, e = lay.pca_cell_start[cc + 1]; k < e; k += 32)
                {
                    float2 fr = lay.pca_frac[k];
                    float v = bilinear(ndf, cell, fr.x, fr.y);
                    uint32_t idx = lay.pca_index[k];
                    if(better(v, idx, best_v, best_i))
                    {
                        best_v = v;
                        best_i = idx;
                    }
                }
            }
        }
    }
    block_argmax(best_v, best_i, sv, si);
    if(threadIdx.x == 0)
    {
        if(best_v > v0 && best_i < (uint32_t)kPcaSamples)
        {
            float4 d = lay.pca_dir[best_i];
            sh_n[0] = d.x;
            sh_n[1] = d.y;
            sh_n[2] = d.z;
        }
        else
        {
            sh_n[0] = 0.0f;
            sh_n[1] = 0.0f;
            sh_n[2] = 1.0f;
        }
    }
    __syncthreads();
    const float n[3] = { sh_n[0], sh_n[1], sh_n[2] };

    // tangent search (pipeline.cc:604-628): Matrix3::makeBasis (matrix3.hh:99-108)
    // then 512 steps of rotateTangentPlane (matrix3.hh:133-137), one thread per
    // vector component (the recurrence does not mix components)
    if(threadIdx.x < 3)
    {
        // d0 = (1,0,0) x n, d1 = (0,1,0) x n (vector3.hh:102-104)
        float d0[3] = { sub(mul(0.0f, n[2]), mul(0.0f, n[1])), sub(mul(0.0f, n[0]), mul(1.0f, n[2])),
                        sub(mul(1.0f, n[1]), mul(0.0f, n[0])) };
        float d1[3] = { sub(mul(1.0f, n[2]), mul(0.0f, n[1])), sub(mul(0.0f, n[0]), mul(0.0f, n[2])),
                        sub(mul(0.0f, n[1]), mul(1.0f, n[0])) };
        float l0 = dot3(d0, d0), l1 = dot3(d1, d1);
        float c0v[3];
        if(l0 > l1)
        {
            float r = dvd(1.0f, __fsqrt_rn(l0));
            c0v[0] = mul(d0[0], r); c0v[1] = mul(d0[1], r); c0v[2] = mul(d0[2], r);
        }
        else
        {
            float r = dvd(1.0f, __fsqrt_rn(l1));
            c0v[0] = mul(d1[0], r); c0v[1] = mul(d1[1], r); c0v[2] = mul(d1[2], r);
        }
        // c1 = n x c0
        float c1v[3] = { sub(mul(n[1], c0v[2]), mul(n[2], c0v[1])), sub(mul(n[2], c0v[0]), mul(n[0], c0v[2])),
                         sub(mul(n[0], c0v[1]), mul(n[1], c0v[0])) };
        const int j = threadIdx.x;
        float a = c0v[j], b = c1v[j];
        const float rs = lay.rot_s, rc = lay.rot_c, nrs = -lay.rot_s;
        for(int k = 0; k < kTangentSteps; ++k)
        {
            tan_seq[j][k] = a;
            float a2 = add(mul(rc, a), mul(rs, b));
            b = add(mul(nrs, a2), mul(rc, b));
            a = a2;
        }
    }
    __syncthreads();
    float tv = 0.0f;
    uint32_t ti = 0xffffffffu;
    for(uint32_t k = threadIdx.x; k < (uint32_t)kTangentSteps; k += kFinishThreads)
    {
        const float d[3] = { tan_seq[0][k], tan_seq[1][k], tan_seq[2][k] };
        float v = pca_value(ndf, d);
        if(v > 0.0f && better(v, k, tv, ti))   // strictly above the initial 0 (pipeline.cc:613-617)
        {
            tv = v;
            ti = k;
        }
    }
    block_argmax(tv, ti, sv, si);
    if(threadIdx.x == 0)
    {
        float bt[3];
        if(ti != 0xffffffffu && tv > 0.0f)
        {
            bt[0] = tan_seq[0][ti];
            bt[1] = tan_seq[1][ti];
            bt[2] = tan_seq[2][ti];
        }
        else
        {
            bt[0] = 1.0f;
            bt[1] = 0.0f;
            bt[2] = 0.0f;
        }
        // B = (bt x n, bt, n) (pipeline.cc:626-627)
        sh_B[0] = sub(mul(bt[1], n[2]), mul(bt[2], n[1]));
        sh_B[1] = sub(mul(bt[2], n[0]), mul(bt[0], n[2]));
        sh_B[2] = sub(mul(bt[0], n[1]), mul(bt[1], n[0]));
        sh_B[3] = bt[0];
        sh_B[4] = bt[1];
        sh_B[5] = bt[2];
        sh_B[6] = n[0];
        sh_B[7] = n[1];
        sh_B[8] = n[2];
        if(info)
        {
            float* o = info + 8 * t;
            o[0] = ndf_denom;
            o[1] = n[0]; o[2] = n[1]; o[3] = n[2];
            o[4] = bt[0]; o[5] = bt[1]; o[6] = bt[2];
            o[7] = best_v > v0 ? best_v : v0;
        }
    }
    __syncthreads();

    // SGGX projection (pipeline.cc:639, SGGXProjectIntegrand :175-189)
    double px = 0.0, py = 0.0, pz = 0.0;
    for(uint32_t s = threadIdx.x; s < (uint32_t)kProjSamples; s += kFinishThreads)
    {
        float4 dd = lay.proj_dir[s];
        if(dd.z <= 0.0f)
            continue;
        const float d[3] = { dd.x, dd.y, dd.z };
        float2 fr = lay.proj_frac[s];
        float v = bilinear(ndf, lay.proj_cell[s], fr.x, fr.y);
        px += (double)mul(fabsf(dot3(d, sh_B + 0)), v);
        py += (double)mul(fabsf(dot3(d, sh_B + 3)), v);
        pz += (double)mul(fabsf(dot3(d, sh_B + 6)), v);
    }
    const float tx = (float)block_sum(px, sd);
    const float ty = (float)block_sum(py, sd);
    const float tz = (float)block_sum(pz, sd);
    if(threadIdx.x == 0)
    {
        // ndf_norm * (total / (samples * pdf)); Vector3 / float multiplies by the reciprocal
        const float rden = dvd(1.0f, mul((float)kProjSamples, lay.pdf));
        const float sx = mul(ndf_norm, mul(tx, rden)), sy = mul(ndf_norm, mul(ty, rden)),
                    sz = mul(ndf_norm, mul(tz, rden));
        // Matrix3::decompose (matrix3.hh:311-332)
        const float* C = sh_B;
        float s0 = __fsqrt_rn(dot3(C, C)), s1 = __fsqrt_rn(dot3(C + 3, C + 3)), s2 = __fsqrt_rn(dot3(C + 6, C + 6));
        float m20 = dvd(C[6], s2);
        float e0, e1, e2;
        if(m20 >= 0.9999f)
        {
            e0 = 0.0f;
            e1 = kPi * 0.5f;
            e2 = atan2f(C[1], C[4]);
        }
        else if(m20 <= -0.9999f)
        {
            e0 = 0.0f;
            e1 = -kPi * 0.5f;
            e2 = atan2f(C[1], C[4]);
        }
        else
        {
            e0 = atan2f(-C[7], C[8]);
            e1 = asinf(m20);
            e2 = atan2f(dvd(-C[3], s1), dvd(C[0], s0));
        }
        float* o = init + 7 * t;
        o[0] = dvd(sx, sz);
        o[1] = dvd(sy, sz);
        o[2] = ndf_denom;
        o[3] = 0.0f;
        o[4] = e0;
        o[5] = e1;
        o[6] = e2;
    }
}

} // namespace

cudaError_t launch_ndf_operator(const InitLayout& lay, const MeshDevice& mesh, const float* ndf_dirs,
                                const float* row_normals, double ndf_scale, int32_t* light_tri, float* light_bary,
                                cudaStream_t stream)
{
    size_t ms = mesh_smem_bytes(lay.L, mesh.ntri, mesh.nedge);
    locate_lights_kernel<<<(kNdfSamples + 255) / 256, 256, ms, stream>>>(mesh, lay.L, ndf_dirs, light_tri, light_bary);
    cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
        return e;
    size_t smem = sizeof(double) * lay.N + ms;
    e = cudaFuncSetAttribute(ndf_operator_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(e != cudaSuccess)
        return e;
    ndf_operator_kernel<<<lay.ndf_rows, 256, smem, stream>>>(mesh, lay.L, lay.N, lay.k_pad, ndf_dirs, row_normals,
                                                             light_tri, light_bary, ndf_scale, lay.ndf_op);
    return cudaGetLastError();
}

cudaError_t launch_init_finish(const InitLayout& lay, const float* ndf_rows, uint32_t ldr, uint64_t texels,
                               float* init_params, float* init_info, float* ndf_out, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    init_finish_kernel<<<(unsigned)texels, kFinishThreads, 0, stream>>>(lay, ndf_rows, ldr, init_params, init_info,
                                                                        ndf_out);
    return cudaGetLastError();
}

} // namespace svf
