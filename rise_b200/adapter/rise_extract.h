// rise_extract.h -- the RISE side of the drop-in boundary: reads a RISE scene
// (RISE::IScene, src/Library/Interfaces/IScene.h) through its interfaces into
// the plain description the rtb200 C ABI (include/rtb200.h) takes, and
// uploads it.  Compiled inside a RISE build (against src/Library), not into
// librtb200.
//
// What is read, and from where:
//  * objects: IObjectManager::EnumerateObjects; each object's geometry
//    through IGeometry::TessellateToMesh (Interfaces/IGeometry.h:74: per-corner
//    positions and normals) moved to world space by the object's
//    ITransformable::GetFinalTransformMatrix (normals by the inverse
//    transpose); meshes whose corner normals all equal their face normals
//    are shaded flat; the double-sided flag of TriangleMeshGeometryIndexed;
//  * materials: LambertianMaterial (reflectance painter), LambertianLuminaire
//    (its LambertianEmitter's exitance painter x scale / pi as radiance, and
//    the reflective material below it), GGXMaterial (rs painter, isotropic
//    alpha, ior / extinction scalar painters per wavelength),
//    DielectricMaterial (ior per wavelength, the scattering exponent);
//  * painters: SpectralColorPainter as its SpectralPacket bins exactly,
//    UniformColorPainter as the albedo uplift of its RGB colour, any other
//    painter sampled per nanometre (GetColorNM) into a 1 nm packet;
//  * the camera: its location, and the directions ICamera::GenerateRay gives
//    through the film's centre and top edge (a pinhole's look-at, up and
//    field of view);
//  * the global radiance map (RadianceMap): a uniform painter as a uniform
//    sky, a texture painter as an image environment read back texel by
//    texel through the painter's own lookups, with its scale and rotation.
// Anything else (other geometry kinds that do not tessellate, other
// materials, lights other than luminaries) is reported, not guessed.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "rtb200.h"

namespace RISE {
class IScene;
}

namespace rtb200_rise {

struct Spectrum {
    int kind = 0;                 // 0: packet (begin, end, amps); 1: RGB sigmoid (coeffs); 2: 81-point grid
    float begin = 380.0f, end = 780.0f;
    std::vector<float> amps;      // packet bins or grid values
    double coeffs[4] = {0, 0, 0, 1};
};

struct Mesh {
    std::vector<float> xyz;       // 3 per corner, world space
    std::vector<float> nrm;       // 3 per corner, or empty (flat shading)
    int32_t material = 0;
    int32_t double_sided = 1;
};

struct EnvImage {
    int width = 0, height = 0;
    std::vector<float> rgb;       // width x height x 3, rows top to bottom
    float scale = 1.0f;
    float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
};

struct Scene {
    std::vector<Spectrum> spectra;
    std::vector<rtb200_material> materials;
    std::vector<Mesh> meshes;
    int32_t env_spectrum = -1, env_visible = 1;
    EnvImage env_image;           // width 0: none
    float cam_pos[3] = {0, 0, 0}, cam_look[3] = {0, 0, 1}, cam_up[3] = {0, 1, 0};
    float fov_deg = 45.0f;
    int32_t width = 0, height = 0;
    std::vector<std::string> refused;   // what could not be read
};

// Reads `scene`; false (with reasons in out.refused) when something on this
// path could not be read.
bool ExtractScene(const RISE::IScene& scene, Scene& out);

// Adds everything to an uncommitted rtb200 scene; an RTB200_* status.
int UploadScene(const Scene& in, rtb200_scene* out);

}  // namespace rtb200_rise
