// pt_api.cpp -- C ABI of the spectral path tracer's scene side: spectra,
// materials, the sky, and the shading tables uploaded at commit
// (include/rtb200.h).  Jobs and engines live in engine.cpp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cie1931.h"
#include "core.h"
#include "env_map.h"
#include "ggx_tables.h"
#include "pathtrace.h"

namespace rtb200 {

namespace {

template <class T>
int Upload(rtb200_ctx* ctx, T** dst, const std::vector<T>& src, size_t& total)
{
    *dst = nullptr;
    if (src.empty()) return RTB200_OK;
    void* p = nullptr;
    int rc = DevAlloc(ctx, &p, src.size() * sizeof(T));
    if (rc) return rc;
    if (cudaMemcpy(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) {
        DevFree(ctx, p, src.size() * sizeof(T));
        return CudaCheck(ctx, cudaGetLastError(), "shading upload");
    }
    total += src.size() * sizeof(T);
    *dst = (T*)p;
    return RTB200_OK;
}

// Light BVH over the luminaries (LightBVH::Build / BuildRecursive,
// Lights/LightBVH.cpp:219-421): each luminary is a primitive with its
// bounding box (degenerate axes widened by 1e-12, BoundingBox::EnsureBoxHasVolume)
// and its selection power; a node holds the union box and the summed power;
// a node of several primitives splits them on the widest axis of their box
// centres at the power-weighted mean centre (std::partition; the middle
// index when one side is empty or the extent is below 1e-10); nodes in
// preorder.  Luminaries are area emitters, whose cones are full spheres.
struct LightPrim {
    double lo[3], hi[3], c[3];
    double power;
    int light;
};

int BuildLightNodes(std::vector<LightPrim>& prims, int start, int end, int& pos, std::vector<PtLightNode>& nodes,
                    std::vector<PtLight>& lights)
{
    const int idx = (int)nodes.size();
    nodes.emplace_back();
    PtLightNode n{};
    double lo[3], hi[3], power = prims[start].power;
    for (int k = 0; k < 3; ++k) { lo[k] = prims[start].lo[k]; hi[k] = prims[start].hi[k]; }
    for (int i = start + 1; i < end; ++i) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], prims[i].lo[k]); hi[k] = std::max(hi[k], prims[i].hi[k]); }
        power += prims[i].power;
    }
    for (int k = 0; k < 3; ++k) { n.lo[k] = (float)lo[k]; n.hi[k] = (float)hi[k]; }
    n.power = (float)power;
    n.count = end - start;
    n.start = pos;
    if (end - start == 1) {
        n.light = prims[start].light;
        lights[n.light].bvh_pos = pos++;
        nodes[idx] = n;
        return idx;
    }
    double clo[3], chi[3];
    for (int k = 0; k < 3; ++k) clo[k] = chi[k] = prims[start].c[k];
    for (int i = start + 1; i < end; ++i)
        for (int k = 0; k < 3; ++k) { clo[k] = std::min(clo[k], prims[i].c[k]); chi[k] = std::max(chi[k], prims[i].c[k]); }
    const double ex[3] = {chi[0] - clo[0], chi[1] - clo[1], chi[2] - clo[2]};
    int axis = 0;
    if (ex[1] > ex[0]) axis = 1;
    if (ex[2] > (axis == 0 ? ex[0] : ex[1])) axis = 2;
    int mid;
    if (ex[axis] < 1e-10) {
        mid = start + (end - start) / 2;
    } else {
        double ws = 0.0, tp = 0.0;
        for (int i = start; i < end; ++i) { ws += prims[i].c[axis] * prims[i].power; tp += prims[i].power; }
        const double split = tp > 0.0 ? ws / tp : 0.5 * (clo[axis] + chi[axis]);
        auto it = std::partition(prims.begin() + start, prims.begin() + end,
                                 [&](const LightPrim& p) { return p.c[axis] < split; });
        mid = (int)(it - prims.begin());
        if (mid == start || mid == end) mid = start + (end - start) / 2;
    }
    nodes[idx] = n;
    BuildLightNodes(prims, start, mid, pos, nodes, lights);
    nodes[idx].right = (int)nodes.size();
    BuildLightNodes(prims, mid, end, pos, nodes, lights);
    return idx;
}

// Walker's alias table by Vose's algorithm (Utilities/AliasTable.h:34-101):
// weights scaled so each entry's fair share is 1, entries below 1 ("small")
// and at or above ("large") kept on stacks; the top small entry keeps its
// scaled weight as its threshold and takes the top large entry as its alias,
// whose weight gives up the difference; leftovers keep themselves.  The same
// stack order as the reference, so a number maps to the same luminary.
std::vector<PtLightAlias> BuildAlias(const std::vector<double>& w)
{
    const size_t n = w.size();
    std::vector<PtLightAlias> out(n);
    double total = 0.0;
    for (double x : w) total += x;
    if (n == 0 || !(total > 0.0)) return out;
    std::vector<double> scaled(n), prob(n, 1.0);
    std::vector<unsigned> alias(n);
    std::vector<unsigned> small, large;
    for (size_t i = 0; i < n; ++i) {
        scaled[i] = w[i] / total * (double)n;
        alias[i] = (unsigned)i;
        (scaled[i] < 1.0 ? small : large).push_back((unsigned)i);
    }
    while (!small.empty() && !large.empty()) {
        const unsigned sm = small.back(), lg = large.back();
        small.pop_back();
        large.pop_back();
        prob[sm] = scaled[sm];
        alias[sm] = lg;
        scaled[lg] = (scaled[lg] + scaled[sm]) - 1.0;
        (scaled[lg] < 1.0 ? small : large).push_back(lg);
    }
    for (size_t i = 0; i < n; ++i) out[i] = PtLightAlias{(float)prob[i], (int)alias[i]};
    return out;
}

}  // namespace

// The image environment as one device block: the PtEnvMap descriptor, its
// texels, the sampling tables and the RGB uplift table, 16-byte aligned.
int UploadEnv(rtb200_scene* s, size_t& total)
{
    rtb200_ctx* ctx = s->ctx;
    const std::vector<float>& up = UpliftTable();
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t o_tex = al(sizeof(PtEnvMap));
    const size_t o_marg = o_tex + al(s->env_texels.size() * sizeof(float4));
    const size_t o_cond = o_marg + al(s->env_marginal.size() * sizeof(float));
    const size_t o_up = o_cond + al(s->env_conditional.size() * sizeof(float));
    const size_t bytes = o_up + al(up.size() * sizeof(float));
    std::vector<unsigned char> host(bytes, 0);
    void* d = nullptr;
    int rc = DevAlloc(ctx, &d, bytes);
    if (rc) return rc;
    unsigned char* base = (unsigned char*)d;
    PtEnvMap E{};
    E.texels = (const float4*)(base + o_tex);
    E.width = s->env_w;
    E.height = s->env_h;
    std::memcpy(E.rot, s->env_rot, sizeof(E.rot));
    E.scale = s->env_scale;
    E.marginal = (const float*)(base + o_marg);
    E.conditional = (const float*)(base + o_cond);
    E.uplift = (const float*)(base + o_up);
    std::memcpy(host.data(), &E, sizeof(E));
    std::memcpy(host.data() + o_tex, s->env_texels.data(), s->env_texels.size() * sizeof(float4));
    std::memcpy(host.data() + o_marg, s->env_marginal.data(), s->env_marginal.size() * sizeof(float));
    std::memcpy(host.data() + o_cond, s->env_conditional.data(), s->env_conditional.size() * sizeof(float));
    std::memcpy(host.data() + o_up, up.data(), up.size() * sizeof(float));
    if (cudaMemcpy(d, host.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
        DevFree(ctx, d, bytes);
        return CudaCheck(ctx, cudaGetLastError(), "environment upload");
    }
    s->d_env = d;
    s->env_bytes = bytes;
    total += bytes;
    return RTB200_OK;
}

int UploadShading(rtb200_scene* s)
{
    rtb200_ctx* ctx = s->ctx;
    if (s->materials.empty()) return RTB200_OK;  // ray casting only
    const size_t nm = s->materials.size();
    for (const PtMaterial& m : s->materials) s->mixed_shading |= m.type != s->materials[0].type;
    s->shade_class = s->mixed_shading ? -1 : s->materials[0].type;
    // GGX conductors: tabulate F_avg(lambda) on the 5 nm grid as an extra
    // spectrum, and make sure the device holds the E_ss / E_avg tables.
    for (PtMaterial& m : s->materials) {
        if (m.type != kMatGGX) continue;
        std::vector<float> favg(RTB200_CIE_COUNT);
        for (int k = 0; k < RTB200_CIE_COUNT; ++k) {
            const double eta = m.eta >= 0 ? s->spectra[(size_t)m.eta * RTB200_CIE_COUNT + k] : m.ior;
            const double kap = m.kappa >= 0 ? s->spectra[(size_t)m.kappa * RTB200_CIE_COUNT + k] : 0.0;
            favg[k] = (float)ConductorFresnelAvg(1.0, eta, kap);
        }
        m.pad = (int)(s->spectra.size() / RTB200_CIE_COUNT);
        s->spectra.insert(s->spectra.end(), favg.begin(), favg.end());
    }
    {
        const GgxTables& gt = GetGgxTables();
        const cudaError_t e = PtSetGgxTables(gt.ess, gt.eavg, gt.msz, gt.mscum, gt.favg_x, gt.favg_w);
        if (e != cudaSuccess) return CudaCheck(ctx, e, "GGX tables");
    }
    for (const auto& mesh : s->meshes)
        if (mesh.material < 0 || (size_t)mesh.material >= nm)
            return SetError(ctx, RTB200_E_INVALID, "mesh material id out of range");
    // Luminaries: one per mesh whose material emits.
    s->lights.clear();
    s->light_tris.clear();
    std::vector<int> meshLight(s->meshes.size(), -1);
    std::vector<double> weight;
    std::vector<LightPrim> boxes;
    for (size_t mi = 0; mi < s->meshes.size(); ++mi) {
        const auto& mesh = s->meshes[mi];
        const PtMaterial& mat = s->materials[mesh.material];
        if (mat.emit < 0 || mesh.count <= 0) continue;
        PtLight L{};
        L.first = (int)s->light_tris.size();
        L.count = (int)mesh.count;
        L.emit = mat.emit;
        double area = 0.0;
        std::vector<double> cum;
        LightPrim box{};
        for (int k = 0; k < 3; ++k) { box.lo[k] = INFINITY; box.hi[k] = -INFINITY; }
        for (int64_t t = mesh.first; t < mesh.first + mesh.count; ++t) {
            const float* v = &s->tri9[9 * (size_t)t];
            for (int j = 0; j < 9; ++j) {
                box.lo[j % 3] = std::min(box.lo[j % 3], (double)v[j]);
                box.hi[j % 3] = std::max(box.hi[j % 3], (double)v[j]);
            }
            PtLightTri lt{};
            for (int k = 0; k < 3; ++k) { lt.v0[k] = v[k]; lt.e1[k] = v[3 + k] - v[k]; lt.e2[k] = v[6 + k] - v[k]; }
            const double cx = (double)lt.e1[1] * lt.e2[2] - (double)lt.e1[2] * lt.e2[1];
            const double cy = (double)lt.e1[2] * lt.e2[0] - (double)lt.e1[0] * lt.e2[2];
            const double cz = (double)lt.e1[0] * lt.e2[1] - (double)lt.e1[1] * lt.e2[0];
            area += 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
            cum.push_back(area);
            s->light_tris.push_back(lt);
        }
        if (!(area > 0.0)) { s->light_tris.resize(L.first); continue; }
        for (size_t k = 0; k < cum.size(); ++k) s->light_tris[L.first + k].cdf = (float)(cum[k] / area);
        s->light_tris[L.first + cum.size() - 1].cdf = 1.0f;
        L.area = (float)area;
        // Selection weight: emitted power, area x mean radiance over 380..780 nm.
        double mean = 0.0;
        for (int k = 0; k < RTB200_CIE_COUNT; ++k) mean += s->spectra[(size_t)mat.emit * RTB200_CIE_COUNT + k];
        mean /= RTB200_CIE_COUNT;
        weight.push_back(area * std::max(mean, 1e-12));
        boxes.push_back(box);
        meshLight[mi] = (int)s->lights.size();
        L.mesh = (int)mi;
        s->lights.push_back(L);
    }
    // Point lights (PointLight.h:49-57, LightSampler.cpp:655-668): the
    // reference weighs a light by its radiant exitance, max(colour x power) x
    // 4 pi for a point light and area x pi x radiance for a luminary.  The
    // luminary weights above omit the common factor pi, so the point light's
    // weight drops it too: max(colour x power) x 4.
    for (const auto& pl : s->point_lights) {
        // A light that emits nothing is left out, as LightSampler::Prepare
        // keeps only lights of positive exitance.
        const double wp = std::max({(double)pl.color[0], (double)pl.color[1], (double)pl.color[2]}) * pl.power * 4.0;
        if (!(wp > 0.0)) continue;
        PtLight L{};
        L.kind = 1;
        L.emit = -1;
        L.mesh = -1;
        L.first = L.count = 0;
        L.le = (float)(0.2126 * pl.color[0] * pl.power + 0.7152 * pl.color[1] * pl.power +
                       0.0722 * pl.color[2] * pl.power);
        for (int k = 0; k < 3; ++k) L.pos[k] = pl.pos[k];
        LightPrim box{};
        for (int k = 0; k < 3; ++k) { box.lo[k] = box.hi[k] = pl.pos[k]; }
        weight.push_back(wp);
        boxes.push_back(box);
        s->lights.push_back(L);
    }
    double wsum = 0.0;
    for (double w : weight) wsum += w;
    for (size_t i = 0; i < s->lights.size(); ++i) s->lights[i].pdf = (float)(weight[i] / wsum);
    s->light_alias = BuildAlias(weight);
    s->light_nodes.clear();
    if (s->lights.size() > 1) {
        std::vector<LightPrim> prims(s->lights.size());
        for (size_t i = 0; i < s->lights.size(); ++i) {
            LightPrim& q = prims[i];
            q = boxes[i];
            for (int k = 0; k < 3; ++k) {
                if (q.lo[k] == q.hi[k]) { q.lo[k] -= 1e-12; q.hi[k] += 1e-12; }
                q.c[k] = 0.5 * (q.lo[k] + q.hi[k]);
            }
            q.power = weight[i];
            q.light = (int)i;
        }
        int pos = 0;
        s->light_nodes.reserve(2 * prims.size());
        BuildLightNodes(prims, 0, (int)prims.size(), pos, s->light_nodes, s->lights);
    }
    // Per-triangle attributes in leaf order.
    const size_t ntri = s->tri_material.size();
    std::vector<int> triMesh(ntri);
    for (size_t mi = 0; mi < s->meshes.size(); ++mi)
        for (int64_t t = s->meshes[mi].first; t < s->meshes[mi].first + s->meshes[mi].count; ++t) triMesh[t] = (int)mi;
    std::vector<PtTriAttr> attr(ntri);
    for (size_t slot = 0; slot < ntri; ++slot) {
        const int mi = triMesh[s->leaf_prims[slot]];
        const auto& mesh = s->meshes[mi];
        attr[slot].mat = (mesh.material & kAttrMatMask) | (mesh.double_sided ? kAttrDoubleSided : 0);
        attr[slot].light = meshLight[mi] >= 0 ? meshLight[mi] : ~mi;
    }
    // Vertex normals in leaf order, unit length, octahedron-encoded; the
    // triangles of meshes without normals keep their face normal.
    s->tri_normals.clear();
    if (!s->tri_smooth.empty()) {
        s->tri_normals.assign(ntri, make_uint4(0, 0, 0, 0));
        for (size_t slot = 0; slot < ntri; ++slot) {
            const uint32_t t = s->leaf_prims[slot];
            if (!s->tri_smooth[t]) continue;
            unsigned q[3];
            for (int j = 0; j < 3; ++j) {
                const float* n = &s->tri_nrm9[9 * (size_t)t + 3 * j];
                const float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                q[j] = OctEncode(n[0] / l, n[1] / l, n[2] / l);
            }
            s->tri_normals[slot] = make_uint4(q[0], q[1], q[2], 0);
            attr[slot].mat |= kAttrSmooth;
        }
    }
    size_t total = 0;
    int rc = Upload(ctx, &s->d_attr, attr, total);
    if (!rc) rc = Upload(ctx, &s->d_mats, s->materials, total);
    // Spectrum table (Spec, pt_device.cuh): headers, then samples.
    std::vector<float> table;
    {
        const size_t nspec = s->spectra.size() / RTB200_CIE_COUNT;
        std::vector<const rtb200_scene::Packet*> packet(nspec, nullptr);
        std::vector<const rtb200_scene::Sigmoid*> sigmoid(nspec, nullptr);
        std::vector<const rtb200_scene::Blackbody*> blackbody(nspec, nullptr);
        for (const auto& q : s->blackbodies) blackbody[q.id] = &q;
        for (const auto& p : s->packets) packet[p.id] = &p;
        for (const auto& q : s->sigmoids) sigmoid[q.id] = &q;
        table.resize(4 * nspec);
        for (size_t id = 0; id < nspec; ++id) {
            const int32_t off = (int32_t)table.size();
            float* h = &table[4 * id];
            if (blackbody[id]) {
                h[0] = -2.0f;
                h[1] = 0.0f;
                h[2] = 1e30f;
                table.push_back(blackbody[id]->t);
                table.push_back(blackbody[id]->scale);
            } else if (sigmoid[id]) {
                h[0] = -1.0f;
                h[1] = 380.0f;
                h[2] = 780.0f;
                table.insert(table.end(), sigmoid[id]->c, sigmoid[id]->c + 4);
            } else if (packet[id]) {
                h[0] = (float)packet[id]->amps.size();
                h[1] = packet[id]->begin;
                h[2] = packet[id]->end;
                table.insert(table.end(), packet[id]->amps.begin(), packet[id]->amps.end());
            } else {
                h[0] = 0.0f;
                h[1] = 380.0f;
                h[2] = 780.0f;
                table.insert(table.end(), s->spectra.begin() + id * RTB200_CIE_COUNT,
                             s->spectra.begin() + (id + 1) * RTB200_CIE_COUNT);
            }
            std::memcpy(&table[4 * id + 3], &off, 4);
        }
    }
    s->spectra_table_bytes = table.size() * sizeof(float);
    if (!rc) rc = Upload(ctx, &s->d_spectra, table, total);
    if (!rc) rc = Upload(ctx, &s->d_lights, s->lights, total);
    if (!rc) rc = Upload(ctx, &s->d_light_tris, s->light_tris, total);
    if (!rc && !s->light_nodes.empty()) rc = Upload(ctx, &s->d_light_nodes, s->light_nodes, total);
    if (!rc && !s->light_alias.empty()) rc = Upload(ctx, &s->d_light_alias, s->light_alias, total);
    if (!rc && !s->tri_normals.empty()) rc = Upload(ctx, &s->d_tri_normals, s->tri_normals, total);
    if (!rc) {
        s->mesh_mat.resize(s->meshes.size());
        for (size_t mi = 0; mi < s->meshes.size(); ++mi) s->mesh_mat[mi] = (int)s->meshes[mi].material;
        rc = Upload(ctx, &s->d_mesh_mat, s->mesh_mat, total);
    }
    if (!rc && s->env_w > 0) rc = UploadEnv(s, total);
    s->shade_bytes = total;
    if (rc) FreeShading(s);
    return rc;
}

void FreeShading(rtb200_scene* s)
{
    rtb200_ctx* ctx = s->ctx;
    DevFree(ctx, s->d_attr, s->tri_material.size() * sizeof(PtTriAttr));
    DevFree(ctx, s->d_mats, s->materials.size() * sizeof(PtMaterial));
    DevFree(ctx, s->d_spectra, s->spectra_table_bytes);
    DevFree(ctx, s->d_lights, s->lights.size() * sizeof(PtLight));
    DevFree(ctx, s->d_light_tris, s->light_tris.size() * sizeof(PtLightTri));
    DevFree(ctx, s->d_light_nodes, s->light_nodes.size() * sizeof(PtLightNode));
    DevFree(ctx, s->d_light_alias, s->light_alias.size() * sizeof(PtLightAlias));
    DevFree(ctx, s->d_tri_normals, s->tri_normals.size() * sizeof(uint4));
    DevFree(ctx, s->d_mesh_mat, s->mesh_mat.size() * sizeof(int));
    s->d_mesh_mat = nullptr;
    DevFree(ctx, s->d_env, s->env_bytes);
    s->d_env = nullptr;
    s->env_bytes = 0;
    s->d_tri_normals = nullptr;
    s->d_light_nodes = nullptr;
    s->d_light_alias = nullptr;
    s->d_attr = nullptr;
    s->d_mats = nullptr;
    s->d_spectra = nullptr;
    s->d_lights = nullptr;
    s->d_light_tris = nullptr;
    s->shade_bytes = 0;
}

}  // namespace rtb200

using namespace rtb200;

extern "C" {

int rtb200_scene_add_spectrum(rtb200_scene* s, const float* values, int32_t* id_out)
{
    if (!s || !values || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    for (int k = 0; k < RTB200_CIE_COUNT; ++k)
        if (!std::isfinite(values[k]) || values[k] < 0.0f)
            return SetError(s->ctx, RTB200_E_INVALID, "spectrum values must be finite and non-negative");
    *id_out = (int32_t)(s->spectra.size() / RTB200_CIE_COUNT);
    s->spectra.insert(s->spectra.end(), values, values + RTB200_CIE_COUNT);
    return RTB200_OK;
}

int rtb200_scene_add_spectral_packet(rtb200_scene* s, float lambda_begin, float lambda_end, int32_t n,
                                     const float* amplitudes, int32_t* id_out)
{
    if (!s || !amplitudes || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    if (n < 1 || n > (1 << 20) || !std::isfinite(lambda_begin) || !std::isfinite(lambda_end) ||
        !(lambda_end > lambda_begin))
        return SetError(s->ctx, RTB200_E_INVALID, "bad spectral packet range");
    for (int32_t k = 0; k < n; ++k)
        if (!std::isfinite(amplitudes[k]) || amplitudes[k] < 0.0f)
            return SetError(s->ctx, RTB200_E_INVALID, "spectrum values must be finite and non-negative");
    rtb200_scene::Packet p;
    p.id = (int32_t)(s->spectra.size() / RTB200_CIE_COUNT);
    p.begin = lambda_begin;
    p.end = lambda_end;
    p.amps.assign(amplitudes, amplitudes + n);
    // Grid samples for the host's uses (conductor Fresnel averages, light
    // selection weights), the packet's own value at each grid wavelength.
    for (int k = 0; k < RTB200_CIE_COUNT; ++k) {
        const double nm = 380.0 + 5.0 * k;
        float v = 0.0f;
        if (nm >= lambda_begin && nm <= lambda_end)
            v = p.amps[std::min((int)((nm - lambda_begin) * n / ((double)lambda_end - lambda_begin)), n - 1)];
        s->spectra.push_back(v);
    }
    *id_out = p.id;
    s->packets.push_back(std::move(p));
    return RTB200_OK;
}

namespace {
// Planck's radiation function as the reference writes it
// (BlackBodyPainter::IntensityForWavelength, BlackBodyPainter.cpp:26-43),
// wavelength in metres.
double Planck(double t, double lambda)
{
    const double c = 2.99792458e8, h = 6.6260755e-34, k = 1.380658e-23;
    const double c1 = 2.0 * 3.14159265358979323846 * h * (c * c), c2 = (h * c) / k;
    return c1 / std::pow(lambda, 5.0) * (1.0 / (std::exp(c2 / (lambda * t)) - 1.0));
}
}  // namespace

int rtb200_scene_add_blackbody(rtb200_scene* s, double temperature, double scale, int32_t normalize, int32_t* id_out)
{
    if (!s || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    if (!(temperature > 0.0) || !std::isfinite(temperature) || !(scale >= 0.0) || !std::isfinite(scale))
        return SetError(s->ctx, RTB200_E_INVALID, "bad black body");
    // With normalize, the scale is divided by the function's value at
    // 0.0029 / T metres (BlackBodyPainter::RegenerateData, :163-168, with
    // PeakNMFromTemperature, :60-63).
    if (normalize) scale /= Planck(temperature, 0.0029 / temperature);
    rtb200_scene::Blackbody q{(int32_t)(s->spectra.size() / RTB200_CIE_COUNT), (float)temperature, (float)scale};
    for (int k = 0; k < RTB200_CIE_COUNT; ++k)
        s->spectra.push_back((float)((double)q.scale * Planck((double)q.t, (380.0 + 5.0 * k) * 1e-9)));
    *id_out = q.id;
    s->blackbodies.push_back(q);
    return RTB200_OK;
}

int rtb200_scene_add_point_light(rtb200_scene* s, const float* position, const float* color, float power)
{
    if (!s || !position || !color) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(position[k]) || !std::isfinite(color[k]) || color[k] < 0.0f)
            return SetError(s->ctx, RTB200_E_INVALID, "bad point light");
    if (!std::isfinite(power) || power < 0.0f) return SetError(s->ctx, RTB200_E_INVALID, "bad point light");
    rtb200_scene::PointLight pl;
    for (int k = 0; k < 3; ++k) { pl.pos[k] = position[k]; pl.color[k] = color[k]; }
    pl.power = power;
    s->point_lights.push_back(pl);
    return RTB200_OK;
}

int rtb200_scene_add_rgb_spectrum(rtb200_scene* s, const double* cs, int32_t* id_out)
{
    if (!s || !cs || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    for (int k = 0; k < 4; ++k)
        if (!std::isfinite(cs[k])) return SetError(s->ctx, RTB200_E_INVALID, "sigmoid coefficients must be finite");
    if (cs[3] < 0.0) return SetError(s->ctx, RTB200_E_INVALID, "spectrum scale must be non-negative");
    rtb200_scene::Sigmoid q;
    q.id = (int32_t)(s->spectra.size() / RTB200_CIE_COUNT);
    for (int k = 0; k < 4; ++k) q.c[k] = (float)cs[k];
    // Grid samples for the host's uses, as the device evaluates the spectrum.
    for (int k = 0; k < RTB200_CIE_COUNT; ++k) {
        const double t = (5.0 * k) / 400.0;
        const double x = (double)q.c[0] * t * t + (double)q.c[1] * t + (double)q.c[2];
        s->spectra.push_back((float)((double)q.c[3] * (0.5 + x / (2.0 * std::sqrt(1.0 + x * x)))));
    }
    *id_out = q.id;
    s->sigmoids.push_back(q);
    return RTB200_OK;
}

int rtb200_scene_add_material(rtb200_scene* s, const rtb200_material* m, int32_t* id_out)
{
    if (!s || !m || !id_out) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    const int nspec = (int)(s->spectra.size() / RTB200_CIE_COUNT);
    auto okSpec = [&](int id) { return id >= -1 && id < nspec; };
    if (m->type < RTB200_MAT_LAMBERTIAN || m->type > RTB200_MAT_DIELECTRIC || !okSpec(m->reflectance) ||
        !okSpec(m->emission) || !okSpec(m->eta) || !okSpec(m->kappa))
        return SetError(s->ctx, RTB200_E_INVALID, "bad material");
    PtMaterial pm{};
    pm.type = m->type;
    pm.refl = m->reflectance;
    pm.emit = m->emission;
    pm.eta = m->eta;
    pm.kappa = m->kappa;
    pm.alpha = m->alpha;
    pm.ior = m->ior;
    pm.pad = -1;   // conductor Fresnel average spectrum, built at commit
    *id_out = (int32_t)s->materials.size();
    s->materials.push_back(pm);
    return RTB200_OK;
}

int rtb200_scene_set_environment_map(rtb200_scene* s, const float* rgb, int32_t width, int32_t height, float scale,
                                     const float* orientation_deg, int32_t visible)
{
    if (!s) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    if (!rgb || width <= 0 || height <= 0 || (int64_t)width * height > (1ll << 26) || !std::isfinite(scale) ||
        scale < 0.0f)
        return SetError(s->ctx, RTB200_E_INVALID, "bad environment map");
    const size_t n = (size_t)width * height;
    std::vector<float4> tex(n);
    for (size_t i = 0; i < n; ++i) {
        const float r = rgb[3 * i], gg = rgb[3 * i + 1], b = rgb[3 * i + 2];
        if (!std::isfinite(r) || !std::isfinite(gg) || !std::isfinite(b))
            return SetError(s->ctx, RTB200_E_INVALID, "environment map holds a non-finite texel");
        tex[i] = make_float4(r, gg, b, 0.0f);
    }
    double orient[3] = {0.0, 0.0, 0.0};
    if (orientation_deg)
        for (int k = 0; k < 3; ++k) orient[k] = (double)orientation_deg[k] * (3.14159265358979323846 / 180.0);
    s->env_texels.swap(tex);
    s->env_w = width;
    s->env_h = height;
    s->env_scale = scale;
    EnvRotation(orient, s->env_rot);
    BuildEnvTables(s->env_texels, width, height, scale, s->env_marginal, s->env_conditional);
    s->env = -1;
    s->env_visible = visible ? 1 : 0;
    return RTB200_OK;
}

int rtb200_scene_set_environment_rotation(rtb200_scene* s, const float* rot9)
{
    if (!s || !rot9) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    if (s->env_w <= 0) return SetError(s->ctx, RTB200_E_INVALID, "scene has no image environment");
    for (int k = 0; k < 9; ++k)
        if (!std::isfinite(rot9[k])) return SetError(s->ctx, RTB200_E_INVALID, "bad environment rotation");
    std::copy(rot9, rot9 + 9, s->env_rot);
    return RTB200_OK;
}

int rtb200_scene_set_environment(rtb200_scene* s, int32_t spectrum, int32_t visible)
{
    if (!s) return RTB200_E_INVALID;
    std::lock_guard<std::mutex> g(s->ctx->mu);
    if (s->committed) return SetError(s->ctx, RTB200_E_INVALID, "scene already committed");
    if (spectrum < -1 || spectrum >= (int32_t)(s->spectra.size() / RTB200_CIE_COUNT))
        return SetError(s->ctx, RTB200_E_INVALID, "bad environment spectrum");
    s->env = spectrum;
    s->env_visible = visible ? 1 : 0;
    s->env_texels.clear();
    s->env_w = s->env_h = 0;
    return RTB200_OK;
}


}  // extern "C"
