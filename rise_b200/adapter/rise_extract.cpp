// rise_extract.cpp -- reads a RISE scene into the rtb200 description (see
// rise_extract.h).  Built inside a RISE tree: the includes are the
// reference's own headers under src/Library.
#include "rise_extract.h"

#include <cmath>
#include <map>

#include "Cameras/PinholeCamera.h"
#include "Geometry/TriangleMeshGeometry.h"
#include "Geometry/TriangleMeshGeometryIndexed.h"
#include "Interfaces/ICamera.h"
#include "Interfaces/IEnumCallback.h"
#include "Interfaces/IFilm.h"
#include "Interfaces/IGeometry.h"
#include "Interfaces/IObjectManager.h"
#include "Interfaces/IObjectPriv.h"
#include "Interfaces/IPainter.h"
#include "Interfaces/IScalarPainter.h"
#include "Interfaces/IScene.h"
#include "Intersection/RayIntersectionGeometric.h"
#include "Materials/DielectricMaterial.h"
#include "Materials/GGXMaterial.h"
#include "Materials/LambertianBRDF.h"
#include "Materials/LambertianEmitter.h"
#include "Materials/LambertianLuminaireMaterial.h"
#include "Materials/LambertianMaterial.h"
#include "Painters/SpectralColorPainter.h"
#include "Painters/TexturePainter.h"
#include "Painters/UniformColorPainter.h"
#include "Polygon.h"
#include "Rendering/RadianceMap.h"
#include "Utilities/RandomNumbers.h"
#include "Utilities/RuntimeContext.h"

using namespace RISE;
using namespace RISE::Implementation;

namespace rtb200_rise {

namespace {

// Protected state the scene's classes keep without accessors; a RISE build
// that adopts this adapter would add getters instead.  Pointers to the
// members are formed through derived classes, as the language allows.
struct MeshAccess : public TriangleMeshGeometryIndexed {
    static bool DoubleSided(const TriangleMeshGeometryIndexed& g) { return g.*(&MeshAccess::bDoubleSided); }
};
struct SoupAccess : public TriangleMeshGeometry {
    static bool DoubleSided(const TriangleMeshGeometry& g) { return g.*(&SoupAccess::bDoubleSided); }
};
struct EmitterAccess : public LambertianEmitter {
    static const IPainter* Painter(const LambertianEmitter& e) { return e.*(&EmitterAccess::pRadEx); }
    static Scalar Scale(const LambertianEmitter& e) { return e.*(&EmitterAccess::scale); }
};
struct TextureAccess : public TexturePainter {
    static const IRasterImageAccessor* Accessor(const TexturePainter& p) { return p.*(&TextureAccess::pRIA); }
};

RayIntersectionGeometric Probe()
{
    return RayIntersectionGeometric(Ray(), nullRasterizerState);
}

struct Builder {
    Scene& out;

    // A painter's spectrum (times `mul`), as its packet, its colour's
    // uplift or 1 nm samples.
    int32_t SpectrumOf(const IPainter& p, double mul = 1.0)
    {
        const auto key = std::make_pair((const void*)&p, mul);
        for (const auto& kv : cache)
            if (kv.first == key) return kv.second;
        Spectrum s;
        RayIntersectionGeometric ri = Probe();
        if (const SpectralColorPainter* sp = dynamic_cast<const SpectralColorPainter*>(&p)) {
            const SpectralPacket pk = sp->GetSpectrum(ri);
            s.kind = 0;
            s.begin = (float)pk.minLambda();
            s.end = (float)pk.maxLambda();
            for (unsigned i = 0; i < pk.NumBins(); ++i)
                s.amps.push_back((float)(mul * pk.ValueAtNM(pk.minLambda() + (i + 0.5) * pk.deltaLambda())));
        } else if (const UniformColorPainter* up = dynamic_cast<const UniformColorPainter*>(&p)) {
            const RISEPel c = up->GetColor(ri);
            const double rgb[3] = {c.r, c.g, c.b};
            double cs[4];
            s.kind = 1;
            rtb200_rgb_uplift(rgb, RTB200_RGB_ALBEDO, cs);
            for (int k = 0; k < 4; ++k) s.coeffs[k] = cs[k];
            s.coeffs[3] *= mul;
        } else {
            s.kind = 0;
            s.begin = 380.0f;
            s.end = 781.0f;
            for (int nm = 380; nm <= 780; ++nm) s.amps.push_back((float)(mul * p.GetColorNM(ri, nm)));
        }
        out.spectra.push_back(s);
        const int32_t id = (int32_t)out.spectra.size() - 1;
        cache.push_back({key, id});
        return id;
    }
    std::vector<std::pair<std::pair<const void*, double>, int32_t>> cache;

    // A physical scalar on the 5 nm grid.
    int32_t ScalarSpectrum(const IScalarPainter& p, bool* constant, double* first)
    {
        RayIntersectionGeometric ri = Probe();
        Spectrum s;
        s.kind = 2;
        for (int i = 0; i < 81; ++i) s.amps.push_back((float)p.GetValueAtNM(ri, 380.0 + 5.0 * i));
        bool c = true;
        for (float v : s.amps) c = c && v == s.amps[0];
        if (constant) *constant = c;
        if (first) *first = p.GetValueAtNM(ri, 550.0);
        out.spectra.push_back(s);
        return (int32_t)out.spectra.size() - 1;
    }

    std::map<const IMaterial*, int32_t> materials;

    int32_t MaterialOf(const IMaterial* m)
    {
        auto it = materials.find(m);
        if (it != materials.end()) return it->second;
        rtb200_material r{};
        r.reflectance = r.emission = r.eta = r.kappa = -1;
        r.ior = 1.5f;
        bool ok = true;
        if (const LambertianLuminaireMaterial* lum = dynamic_cast<const LambertianLuminaireMaterial*>(m)) {
            // An emitter over a base material, whose BSDF the luminaire
            // passes through (a Lambertian one, or none for "none").
            r.type = RTB200_MAT_LAMBERTIAN;
            const LambertianEmitter* em = dynamic_cast<const LambertianEmitter*>(lum->GetEmitter());
            if (em) {
                // LambertianEmitter::emittedRadianceNM: exitance x scale / pi.
                r.emission = SpectrumOf(*EmitterAccess::Painter(*em), EmitterAccess::Scale(*em) / 3.14159265358979323846);
            } else {
                ok = false;
            }
            if (const LambertianBRDF* lb = dynamic_cast<const LambertianBRDF*>(lum->GetBSDF())) {
                r.reflectance = SpectrumOf(lb->GetReflectance());
            } else if (lum->GetBSDF()) {
                ok = false;
            }
        } else if (const LambertianMaterial* lm = dynamic_cast<const LambertianMaterial*>(m)) {
            r.type = RTB200_MAT_LAMBERTIAN;
            r.reflectance = SpectrumOf(lm->GetReflectance());
        } else if (const GGXMaterial* gm = dynamic_cast<const GGXMaterial*>(m)) {
            RayIntersectionGeometric ri = Probe();
            r.type = RTB200_MAT_GGX;
            r.reflectance = SpectrumOf(gm->GetSpecular());
            r.alpha = (float)gm->GetAlphaX().GetValuesAt(ri).v[0];
            r.eta = ScalarSpectrum(gm->GetIOR(), nullptr, nullptr);
            r.kappa = ScalarSpectrum(gm->GetExtinction(), nullptr, nullptr);
        } else if (const DielectricMaterial* dm = dynamic_cast<const DielectricMaterial*>(m)) {
            RayIntersectionGeometric ri = Probe();
            r.type = RTB200_MAT_DIELECTRIC;
            bool constant = true;
            double n550 = 1.5;
            const int32_t sid = ScalarSpectrum(dm->GetIOR(), &constant, &n550);
            if (constant) r.ior = out.spectra[sid].amps[0];
            else r.eta = sid;
            r.alpha = (float)std::min(1e6, (double)dm->GetScattering().GetValuesAt(ri).v[0]);
        } else {
            ok = false;
        }
        if (!ok) out.refused.push_back("material of a model this path does not draw");
        out.materials.push_back(r);
        return materials[m] = (int32_t)out.materials.size() - 1;
    }
};

struct ObjectWalk : public IEnumCallback<IObjectPriv> {
    Builder* b;
    bool operator()(const IObjectPriv& obj) override
    {
        const IGeometry* g = obj.GetGeometry();
        if (!g) {
            b->out.refused.push_back("object without geometry");
            return true;
        }
        IndexTriangleListType tris;
        VerticesListType verts;
        NormalsListType norms;
        TexCoordsListType coords;
        if (!g->TessellateToMesh(tris, verts, norms, coords, 0) || tris.empty()) {
            b->out.refused.push_back("geometry that does not tessellate to triangles");
            return true;
        }
        const Matrix4 M = obj.GetFinalTransformMatrix();
        const Matrix4 Minv = obj.GetFinalInverseTransformMatrix();
        Mesh mesh;
        mesh.material = obj.GetMaterial() ? b->MaterialOf(obj.GetMaterial()) : 0;
        // The triangle meshes carry a double-sided flag (TriangleMeshGeometry
        // from RAW files, TriangleMeshGeometryIndexed from indexed ones);
        // other tessellated geometry is closed and one-sided.
        if (const TriangleMeshGeometryIndexed* tm = dynamic_cast<const TriangleMeshGeometryIndexed*>(g))
            mesh.double_sided = MeshAccess::DoubleSided(*tm) ? 1 : 0;
        else if (const TriangleMeshGeometry* ts = dynamic_cast<const TriangleMeshGeometry*>(g))
            mesh.double_sided = SoupAccess::DoubleSided(*ts) ? 1 : 0;
        else
            mesh.double_sided = 0;
        bool flat = true;
        for (const IndexedTriangle& t : tris) {
            Point3 p[3];
            for (int k = 0; k < 3; ++k) p[k] = Point3Ops::Transform(M, verts[t.iVertices[k]]);
            const Vector3 fn = Vector3Ops::Normalize(
                Vector3Ops::Cross(Vector3Ops::mkVector3(p[1], p[0]), Vector3Ops::mkVector3(p[2], p[0])));
            for (int k = 0; k < 3; ++k) {
                mesh.xyz.push_back((float)p[k].x);
                mesh.xyz.push_back((float)p[k].y);
                mesh.xyz.push_back((float)p[k].z);
                // Normals go by the inverse transpose of the point transform
                // (which is out_c = sum_r M._rc v_r).
                const Vector3& n0 = norms[t.iNormals[k]];
                const Vector3 n = Vector3Ops::Normalize(Vector3(Minv._00 * n0.x + Minv._01 * n0.y + Minv._02 * n0.z,
                                                                Minv._10 * n0.x + Minv._11 * n0.y + Minv._12 * n0.z,
                                                                Minv._20 * n0.x + Minv._21 * n0.y + Minv._22 * n0.z));
                if (std::fabs(Vector3Ops::Dot(n, fn)) < 1.0 - 1e-9) flat = false;
                mesh.nrm.push_back((float)n.x);
                mesh.nrm.push_back((float)n.y);
                mesh.nrm.push_back((float)n.z);
            }
        }
        if (flat) mesh.nrm.clear();
        b->out.meshes.push_back(std::move(mesh));
        return true;
    }
};

}  // namespace

bool ExtractScene(const IScene& scene, Scene& out)
{
    Builder b{out, {}, {}};
    const IFilm* film = scene.GetFilm();
    if (!film) {
        out.refused.push_back("scene without a film");
        return false;
    }
    out.width = (int32_t)film->GetWidth();
    out.height = (int32_t)film->GetHeight();
    // Camera: location, and the rays through the film's centre and the
    // middle of its top edge (screen y runs up from the bottom row).
    const ICamera* cam = scene.GetCamera();
    if (!cam) {
        out.refused.push_back("scene without a camera");
        return false;
    }
    {
        RandomNumberGenerator rng(1u);
        RuntimeContext rc(rng, RuntimeContext::PASS_NORMAL, false);
        Ray c, top;
        const double w = out.width, h = out.height;
        if (!cam->GenerateRay(rc, c, Point2(w * 0.5, h * 0.5)) || !cam->GenerateRay(rc, top, Point2(w * 0.5, h))) {
            out.refused.push_back("camera that generates no ray through the film centre");
            return false;
        }
        const Point3 o = c.origin;
        const Vector3 f = Vector3Ops::Normalize(c.Dir()), t = Vector3Ops::Normalize(top.Dir());
        // up: the top-edge direction's part orthogonal to the forward one.
        const Vector3 u = Vector3Ops::Normalize(t - f * Vector3Ops::Dot(t, f));
        const double half = std::acos(std::max(-1.0, std::min(1.0, Vector3Ops::Dot(f, t))));
        out.cam_pos[0] = (float)o.x; out.cam_pos[1] = (float)o.y; out.cam_pos[2] = (float)o.z;
        out.cam_look[0] = (float)(o.x + f.x); out.cam_look[1] = (float)(o.y + f.y); out.cam_look[2] = (float)(o.z + f.z);
        out.cam_up[0] = (float)u.x; out.cam_up[1] = (float)u.y; out.cam_up[2] = (float)u.z;
        out.fov_deg = (float)(2.0 * half * 180.0 / 3.14159265358979323846);
    }
    if (const IObjectManager* om = scene.GetObjects()) {
        ObjectWalk walk;
        walk.b = &b;
        om->EnumerateObjects(walk);
    }
    if (const RadianceMap* rm = dynamic_cast<const RadianceMap*>(scene.GetGlobalRadianceMap())) {
        const IPainter& p = rm->GetPainter();
        // RadianceMap::GetRadianceNM turns a world direction by its transform
        // (Vector3Ops::Transform); the rows of that map are its images of the
        // axes.
        const Matrix4& T = rm->GetTransform();
        float rot[9];
        for (int j = 0; j < 3; ++j) {
            const Vector3 e(j == 0, j == 1, j == 2);
            const Vector3 m = Vector3Ops::Transform(T, e);
            rot[0 * 3 + j] = (float)m.x;
            rot[1 * 3 + j] = (float)m.y;
            rot[2 * 3 + j] = (float)m.z;
        }
        if (const TexturePainter* tp = dynamic_cast<const TexturePainter*>(&p)) {
            const IRasterImageAccessor* acc = TextureAccess::Accessor(*tp);
            EnvImage& e = out.env_image;
            e.width = (int)acc->GetWidth();
            e.height = (int)acc->GetHeight();
            e.scale = (float)rm->GetScale();
            std::copy(rot, rot + 9, e.rot);
            // Texel (x, y) read back through the painter at s = (x - 1/2) / W,
            // t = (y - 1/2) / H, where the bilinear lookup lands on it alone.
            RayIntersectionGeometric ri = Probe();
            e.rgb.resize((size_t)e.width * e.height * 3);
            for (int y = 0; y < e.height; ++y)
                for (int x = 0; x < e.width; ++x) {
                    ri.ptCoord = Point2((x - 0.5) / e.width, (y - 0.5) / e.height);
                    const RISEPel c = tp->GetColor(ri);
                    float* o = &e.rgb[3 * ((size_t)y * e.width + x)];
                    o[0] = (float)c.r; o[1] = (float)c.g; o[2] = (float)c.b;
                }
        } else {
            out.env_spectrum = b.SpectrumOf(p, rm->GetScale());
        }
    }
    return out.refused.empty();
}

int UploadScene(const Scene& in, rtb200_scene* s)
{
    std::vector<int32_t> sid(in.spectra.size());
    for (size_t i = 0; i < in.spectra.size(); ++i) {
        const Spectrum& sp = in.spectra[i];
        int rc;
        if (sp.kind == 0) rc = rtb200_scene_add_spectral_packet(s, sp.begin, sp.end, (int32_t)sp.amps.size(),
                                                                 sp.amps.data(), &sid[i]);
        else if (sp.kind == 1) rc = rtb200_scene_add_rgb_spectrum(s, sp.coeffs, &sid[i]);
        else rc = rtb200_scene_add_spectrum(s, sp.amps.data(), &sid[i]);
        if (rc) return rc;
    }
    auto map = [&](int32_t id) { return id < 0 ? id : sid[id]; };
    std::vector<int32_t> mid(in.materials.size());
    for (size_t i = 0; i < in.materials.size(); ++i) {
        rtb200_material m = in.materials[i];
        m.reflectance = map(m.reflectance);
        m.emission = map(m.emission);
        m.eta = map(m.eta);
        m.kappa = map(m.kappa);
        const int rc = rtb200_scene_add_material(s, &m, &mid[i]);
        if (rc) return rc;
    }
    for (const Mesh& m : in.meshes) {
        const int64_t nv = (int64_t)(m.xyz.size() / 3);
        std::vector<uint32_t> tri((size_t)nv);
        for (int64_t i = 0; i < nv; ++i) tri[(size_t)i] = (uint32_t)i;
        int rc;
        if (m.nrm.empty()) {
            rc = rtb200_scene_add_mesh(s, m.xyz.data(), nv, tri.data(), nv / 3, mid[m.material], m.double_sided);
        } else {
            rc = rtb200_scene_add_mesh_normals(s, m.xyz.data(), nv, tri.data(), nv / 3, m.nrm.data(), nv,
                                               tri.data(), mid[m.material], m.double_sided);
        }
        if (rc) return rc;
    }
    int rc = rtb200_scene_set_environment(s, map(in.env_spectrum), in.env_visible);
    if (!rc && in.env_image.width > 0) {
        const EnvImage& e = in.env_image;
        rc = rtb200_scene_set_environment_map(s, e.rgb.data(), e.width, e.height, e.scale, nullptr, in.env_visible);
        if (!rc) rc = rtb200_scene_set_environment_rotation(s, e.rot);
    }
    return rc;
}

}  // namespace rtb200_rise
