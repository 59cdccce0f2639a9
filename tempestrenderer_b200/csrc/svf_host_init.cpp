// svf_host_init.cpp - the default-init tables of a direction layout, built once
// per (directions, mesh) pair: the NDF operator and its tile lists for the
// tcgen05 GEMM, the NDF normalisation weights, the PCA cell and projection
// tables; and the launch of the NDF GEMM over them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/svf.h"
#include "svf_host.h"
#include "svf_internal.h"
#include "svf_btf_file.h"
#include "svf_layout.h"

using namespace svfh;

namespace
{

// Interleaves the bits of x and y (x in the even bits).
uint64_t morton2(uint32_t x, uint32_t y)
{
    uint64_t z = 0;
    for(int b = 0; b < 16; ++b)
        z |= (uint64_t)((x >> b) & 1u) << (2 * b) | (uint64_t)((y >> b) & 1u) << (2 * b + 1);
    return z;
}

// The NDF GEMM's column order: pairs lv = view L + light sorted (stably) by the
// Morton code of their half vector's parabolic coordinates on a 256 x 256 grid,
// so that neighbouring columns reach neighbouring NDF texels.
void half_vector_order(const std::vector<float>& lp, uint32_t L, std::vector<uint32_t>& col_of,
                       std::vector<uint16_t>& col_pos)
{
    const uint32_t N = L * L;
    std::vector<float> w(3 * L);
    for(uint32_t d = 0; d < L; ++d)
        svf::parabolic_to_cartesian_ref(lp[2 * d], lp[2 * d + 1], &w[3 * d]);
    std::vector<uint64_t> code(N);
    const auto q = [](double v) { return (uint32_t)std::min(255.0, std::max(0.0, std::floor((v + 1.0) * 128.0))); };
    for(uint32_t v = 0; v < L; ++v)
        for(uint32_t l = 0; l < L; ++l)
        {
            double h[3] = { (double)w[3 * v] + w[3 * l], (double)w[3 * v + 1] + w[3 * l + 1],
                            (double)w[3 * v + 2] + w[3 * l + 2] };
            const double n = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
            double px = 0.0, py = 0.0;
            if(n > 1e-12)
            {
                const double den = 1.0 + h[2] / n;
                if(den > 1e-12)
                {
                    px = h[0] / n / den;
                    py = h[1] / n / den;
                }
            }
            code[v * L + l] = morton2(q(px), q(py));
        }
    col_of.resize(N);
    for(uint32_t k = 0; k < N; ++k)
        col_of[k] = k;
    std::stable_sort(col_of.begin(), col_of.end(), [&](uint32_t a, uint32_t b) { return code[a] < code[b]; });
    col_pos.resize(N);
    for(uint32_t p = 0; p < N; ++p)
        col_pos[col_of[p]] = (uint16_t)p;
}

} // namespace

namespace svfh
{

// Builds (once per mesh) the default-init tables of a layout, with the given
// mesh or the library's own triangulation.
svf_status prepare_init(svf_ctx* ctx, Layout* lay, const svf_layout_desc* desc, const svf::InitLayout** out)
{
    const uint32_t L = lay->L, N = L * L;
    uint64_t key = 0;   // 0: the library's triangulation
    if(desc->triangles)
    {
        if(desc->triangle_count == 0 || !desc->edges || !desc->edge_angles || desc->edge_count == 0)
            return fail(SVF_EINVAL, "a given mesh needs triangles, edges and edge angles");
        key = fnv1a(desc->triangles, sizeof(uint32_t) * 3 * (size_t)desc->triangle_count);
        key = fnv1a(desc->edges, sizeof(uint32_t) * 3 * (size_t)desc->edge_count, key);
        key = fnv1a(desc->edge_angles, sizeof(float) * 2 * (size_t)desc->edge_count, key) | 1u;
    }
    auto found = lay->inits.find(key);
    if(found != lay->inits.end())
    {
        *out = &found->second->init;
        return SVF_OK;
    }
    std::vector<uint32_t> tris, edges;
    std::vector<float> eang;
    if(desc->triangles)
    {
        tris.assign(desc->triangles, desc->triangles + 3 * (size_t)desc->triangle_count);
        edges.assign(desc->edges, desc->edges + 3 * (size_t)desc->edge_count);
        eang.assign(desc->edge_angles, desc->edge_angles + 2 * (size_t)desc->edge_count);
        for(uint32_t v : tris)
            if(v >= L)
                return fail(SVF_EINVAL, "triangle vertex %u out of range", v);
        for(size_t i = 0; i < edges.size(); i += 3)
            if(edges[i] >= L || edges[i + 1] >= L || edges[i + 2] >= desc->triangle_count)
                return fail(SVF_EINVAL, "edge %zu out of range", i / 3);
    }
    else
    {
        if(!svf::delaunay(lay->lp.data(), L, tris))
            return fail(SVF_EINVAL, "Delaunay triangulation of the directions failed");
        svf::boundary_edges(lay->lp.data(), tris, edges, eang);
    }
    if(!ctx->tables)
    {
        ctx->tables = std::make_unique<svf::InitHostTables>();
        svf::build_init_host_tables(*ctx->tables);
    }
    const svf::InitHostTables& t = *ctx->tables;
    auto data = std::make_unique<InitData>();
    InitData* dd = data.get();
    svf::InitLayout& il = dd->init;
    il.L = L;
    il.N = N;
    il.k_pad = (uint32_t)round_up(N, 8);
    il.ndf_rows = (uint32_t)t.ndf_row_texel.size();
    il.ndf_rows_pad = (uint32_t)round_up(il.ndf_rows, 256);
    SVF_TRY(dd->op.ensure(sizeof(float) * il.ndf_rows_pad * (size_t)il.k_pad));
    SVF_CUDA(cudaMemset(dd->op.p, 0, sizeof(float) * il.ndf_rows_pad * (size_t)il.k_pad));
    // operator rows in Morton order of their NDF texel (a 256-row tile is then a
    // compact block of the texture)
    std::vector<uint32_t> row_order(il.ndf_rows);
    for(uint32_t r = 0; r < il.ndf_rows; ++r)
        row_order[r] = r;
    std::stable_sort(row_order.begin(), row_order.end(), [&](uint32_t a, uint32_t b) {
        const int32_t ta = t.ndf_row_texel[a], tb = t.ndf_row_texel[b];
        return morton2((uint32_t)(ta % svf::kNdfRes), (uint32_t)(ta / svf::kNdfRes)) <
               morton2((uint32_t)(tb % svf::kNdfRes), (uint32_t)(tb / svf::kNdfRes));
    });
    std::vector<int32_t> row_texel(il.ndf_rows);
    std::vector<float> row_normal(3 * (size_t)il.ndf_rows);
    for(uint32_t r = 0; r < il.ndf_rows; ++r)
    {
        row_texel[r] = t.ndf_row_texel[row_order[r]];
        for(int c = 0; c < 3; ++c)
            row_normal[3 * r + c] = t.ndf_row_normal[3 * row_order[r] + c];
    }
    SVF_TRY(upload(dd->row_texel, row_texel));
    SVF_TRY(upload(dd->denom_w, t.denom_w));
    SVF_TRY(upload(dd->pca_cell_id, t.pca_cell_id));
    SVF_TRY(upload(dd->pca_cell_start, t.pca_cell_start));
    SVF_TRY(upload(dd->pca_index, t.pca_index));
    SVF_TRY(upload(dd->pca_frac, t.pca_frac));
    SVF_TRY(upload(dd->pca_dir, t.pca_dir));
    SVF_TRY(upload(dd->proj_dir, t.proj_dir));
    SVF_TRY(upload(dd->proj_frac, t.proj_frac));
    SVF_TRY(upload(dd->proj_cell, t.proj_cell));
    il.ndf_op = dd->op.as<float>();
    il.ndf_row_texel = dd->row_texel.as<int32_t>();
    il.denom_w = dd->denom_w.as<float>();
    il.pca_cells = (uint32_t)t.pca_cell_id.size();
    il.pca_cell_id = dd->pca_cell_id.as<int32_t>();
    il.pca_cell_start = dd->pca_cell_start.as<uint32_t>();
    il.pca_index = dd->pca_index.as<uint32_t>();
    il.pca_frac = dd->pca_frac.as<float2>();
    il.pca_dir = dd->pca_dir.as<float4>();
    il.proj_dir = dd->proj_dir.as<float4>();
    il.proj_frac = dd->proj_frac.as<float2>();
    il.proj_cell = dd->proj_cell.as<int32_t>();
    il.rot_s = t.rot_s;
    il.rot_c = t.rot_c;
    il.pdf = t.pdf;
    il.axis_cell = t.axis_cell;
    il.axis_fx1 = t.axis_frac[0];
    il.axis_fy1 = t.axis_frac[1];

    // the NDF operator, built on the device
    DevBuf d_lp, d_tri, d_edges, d_eang, d_dirs, d_normals, d_ltri, d_lbary;
    SVF_TRY(upload(d_lp, lay->lp));
    SVF_TRY(upload(d_tri, tris));
    SVF_TRY(upload(d_edges, edges));
    SVF_TRY(upload(d_eang, eang));
    SVF_TRY(upload(d_dirs, t.ndf_dirs));
    SVF_TRY(upload(d_normals, row_normal));
    SVF_TRY(d_ltri.ensure(sizeof(int32_t) * svf::kNdfSamples));
    SVF_TRY(d_lbary.ensure(sizeof(float) * 3 * svf::kNdfSamples));
    svf::MeshDevice mesh{ d_lp.as<float>(), d_tri.as<uint32_t>(), (uint32_t)(tris.size() / 3), d_edges.as<uint32_t>(),
                          d_eang.as<float>(), (uint32_t)(edges.size() / 3) };
    SVF_CUDA(svf::launch_ndf_operator(il, mesh, d_dirs.as<float>(), d_normals.as<float>(), t.ndf_scale,
                                      d_ltri.as<int32_t>(), d_lbary.as<float>(), ctx->stream));
    // its non-empty 256 x 64 tiles (columns in half-vector order), packed as the
    // BF16 hi/lo split for the tensor-core GEMM
    std::vector<uint32_t> col_of;
    std::vector<uint16_t> col_pos;
    half_vector_order(lay->lp, L, col_of, col_pos);
    SVF_TRY(upload(dd->col_of, col_of));
    SVF_TRY(upload(dd->col_pos, col_pos));
    il.col_of = dd->col_of.as<uint32_t>();
    il.col_pos = dd->col_pos.as<uint16_t>();
    const uint32_t ktiles = (N + 63) / 64, ntiles = il.ndf_rows_pad / 256;
    DevBuf d_flags;
    SVF_TRY(d_flags.ensure(sizeof(uint32_t) * ktiles * ntiles));
    SVF_CUDA(svf::launch_ndf_tile_flags(il.ndf_op, il.k_pad, il.col_of, N, il.ndf_rows_pad, d_flags.as<uint32_t>(),
                                        ctx->stream));
    std::vector<uint32_t> flags(ktiles * ntiles);
    SVF_CUDA(cudaMemcpyAsync(flags.data(), d_flags.p, sizeof(uint32_t) * flags.size(), cudaMemcpyDeviceToHost,
                             ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<uint32_t> tile_n, tile_kb, tile_start(ntiles + 1, 0);
    for(uint32_t n = 0; n < ntiles; ++n)
    {
        tile_start[n] = (uint32_t)tile_kb.size();
        for(uint32_t kb = 0; kb < ktiles; ++kb)
            if(flags[n * ktiles + kb])
            {
                tile_n.push_back(n);
                tile_kb.push_back(kb);
            }
    }
    tile_start[ntiles] = (uint32_t)tile_kb.size();
    il.packed_tiles = (uint32_t)tile_kb.size();
    if(il.packed_tiles == 0)
    {
        // an operator without a non-zero: one zero tile that no row tile lists
        tile_n.push_back(0);
        tile_kb.push_back(0);
    }
    const uint32_t alloc_tiles = (uint32_t)tile_kb.size();
    DevBuf d_tile_n;
    SVF_TRY(upload(d_tile_n, tile_n));
    SVF_TRY(upload(dd->tile_kb, tile_kb));
    SVF_TRY(upload(dd->tile_start, tile_start));
    SVF_TRY(dd->tile_hi.ensure(sizeof(uint16_t) * 256 * 64 * (size_t)alloc_tiles));
    SVF_TRY(dd->tile_lo.ensure(sizeof(uint16_t) * 256 * 64 * (size_t)alloc_tiles));
    if(il.packed_tiles == 0)
    {
        SVF_CUDA(cudaMemsetAsync(dd->tile_hi.p, 0, sizeof(uint16_t) * 256 * 64, ctx->stream));
        SVF_CUDA(cudaMemsetAsync(dd->tile_lo.p, 0, sizeof(uint16_t) * 256 * 64, ctx->stream));
    }
    else
        SVF_CUDA(svf::launch_ndf_tile_pack(il.ndf_op, il.k_pad, il.col_of, N, d_tile_n.as<uint32_t>(),
                                           dd->tile_kb.as<uint32_t>(), il.packed_tiles, dd->tile_hi.p, dd->tile_lo.p,
                                           ctx->stream));
    il.packed_tiles = alloc_tiles;
    il.nonempty_tiles = tile_start[ntiles];
    il.all_tiles = ktiles * ntiles;
    il.tile_hi = dd->tile_hi.p;
    il.tile_lo = dd->tile_lo.p;
    il.tile_kb = dd->tile_kb.as<uint32_t>();
    il.tile_start = dd->tile_start.as<uint32_t>();
    if(getenv("SVF_DEBUG"))
        fprintf(stderr, "svf: NDF operator L=%u: %u of %u tiles non-empty (%.1f%%)\n", L, tile_start[ntiles],
                ktiles * ntiles, 100.0 * tile_start[ntiles] / (ktiles * ntiles));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = &dd->init;
    lay->inits.emplace(key, std::move(data));
    return SVF_OK;
}

// The NDF rows of `texels` luminance splits (columns in the operator's order) on
// the tensor cores, over the operator's non-empty tiles.
cudaError_t launch_ndf(const svf::InitLayout& il, const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda,
                       float* C, uint32_t ldc, uint32_t* error_flag, cudaStream_t stream)
{
    return svf::launch_ndf_tc_tiles(a_hi, a_lo, texels, lda, il.tile_hi, il.tile_lo, il.ndf_rows_pad, il.k_pad, il.N,
                                    C, ldc, error_flag, stream, il.tile_kb, il.tile_start, il.packed_tiles);
}

} // namespace svfh
