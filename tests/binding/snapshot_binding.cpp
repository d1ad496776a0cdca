// The caller-side binding of the integration guide, compiled against the reference's own headers
// (include/minirender/scene/scene.hpp, render/path_tracer.hpp, render/render_session.hpp) with
// the project's GLM stand-in (tests/binding/glm), and run on a snapshot.
//
// tests/test_binding.py extracts the guide's C++ block into two files: `to_b200.inc` (its
// includes, `B200Snapshot` and `to_b200`) and `render_cli.inc` (the lines that replace
// render_cli.cpp's session, compiled here inside a function that is never called). This program
// builds a SceneSnapshot the way the reference's `make_snapshot` hands it to the path tracer
// (instances with resolved meshes, materials, matrices and textures), converts it with `to_b200`
// and renders the result with the oracle (the FP64 CPU restatement of the reference's path
// tracer, linked as a test library). The test renders the same scene built through the Python
// scene model and requires the two images to be bitwise equal.
//
// The reference defines Image's and Texture's members in its .cpp files, which need libraries
// this image lacks; the few the binding calls are defined below for the test.

#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "to_b200.inc"

#include <minirender/render/render_session.hpp>

namespace minirender {

Image::Image(std::size_t width, std::size_t height)
    : width_(width), height_(height), pixels_(width * height) {}
std::size_t Image::width() const noexcept { return width_; }
std::size_t Image::height() const noexcept { return height_; }
glm::vec3& Image::at(std::size_t x, std::size_t y) { return pixels_[y * width_ + x]; }
const glm::vec3& Image::at(std::size_t x, std::size_t y) const { return pixels_[y * width_ + x]; }
Texture::Texture(Image image, CancellationToken) { levels_.push_back(std::move(image)); }
const Image& Texture::level(std::size_t index) const { return levels_.at(index); }

}  // namespace minirender

// The guide's replacement of render_cli.cpp's session: compiled and linked, not run (it needs a GPU).
[[maybe_unused]] static void render_cli_excerpt(
    const std::shared_ptr<const minirender::SceneSnapshot>& snapshot, const minirender::RenderSettings& render,
    const minirender::IntegratorSettings& integrator, const minirender::SessionSettings& settings) {
#include "render_cli.inc"
    (void)image;
}

extern "C" {
int    or_scene_create(const mr_scene_desc* desc, const mr_bvh_desc* bvh,
                       const mr_integrator_settings* integrator, void** out);
void   or_scene_destroy(void* scene);
int    or_render_rows(void* scene, const mr_render_settings* render, uint64_t row_begin, uint64_t row_end,
                      uint32_t threads, float* rgb, mr_path_statistics* statistics);
size_t or_last_error(char* buffer, size_t capacity);
}

namespace {

using minirender::MeshCorner;
using minirender::MeshData;
using minirender::MeshTriangle;

// A unit quad in the xz plane, facing +y (or -y when `down`), UVs over [0, 1]^2.
std::shared_ptr<const MeshData> quad(bool down) {
    auto mesh       = std::make_shared<MeshData>();
    mesh->positions = {{-1, 0, -1}, {1, 0, -1}, {1, 0, 1}, {-1, 0, 1}};
    const glm::vec3 n(0, down ? -1.0f : 1.0f, 0);
    const glm::vec2 uv[4] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    const int       tris[2][3] = {{0, 3, 2}, {0, 2, 1}};
    for (const auto& t : tris) {
        MeshTriangle tri;
        for (int k = 0; k < 3; ++k) {
            const int i       = down ? t[2 - k] : t[k];
            tri.corners[k]    = MeshCorner{static_cast<std::uint32_t>(i), n, uv[i]};
        }
        mesh->triangles.push_back(tri);
    }
    return mesh;
}

// Translation and per-axis scale, column-major like glm::translate * glm::scale.
glm::mat4 translate_scale(glm::vec3 t, glm::vec3 s) {
    glm::mat4 m(1.0f);
    m[0][0] = s.x;
    m[1][1] = s.y;
    m[2][2] = s.z;
    m[3][0] = t.x;
    m[3][1] = t.y;
    m[3][2] = t.z;
    return m;
}

// The inverse transpose of the scale, in double and stored as float (as Transform::normal_matrix).
glm::mat3 inverse_scale(glm::vec3 s) {
    glm::mat3 m(1.0f);
    m[0][0] = static_cast<float>(1.0 / double(s.x));
    m[1][1] = static_cast<float>(1.0 / double(s.y));
    m[2][2] = static_cast<float>(1.0 / double(s.z));
    return m;
}

std::shared_ptr<const minirender::Texture> texture(std::size_t w, std::size_t h, float seed) {
    minirender::Image image(w, h);
    for (std::size_t y = 0; y < h; ++y) {
        for (std::size_t x = 0; x < w; ++x) {
            const float v = static_cast<float>((x * 7 + y * 13) % 11) / 10.0f;
            image.at(x, y) = glm::vec3(0.2f + 0.6f * v, 0.5f + 0.25f * seed, 0.9f - 0.5f * v);
        }
    }
    return std::make_shared<const minirender::Texture>(std::move(image));
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s out.f32\n", argv[0]);
        return 2;
    }
    minirender::SceneSnapshot s;
    s.camera.position         = glm::vec3(0.3f, 2.5f, 3.0f);
    s.camera.target           = glm::vec3(0.0f, 0.2f, 0.0f);
    s.camera.up               = glm::vec3(0.0f, 1.0f, 0.0f);
    s.camera.vertical_fov_degrees = 50.0f;
    s.camera.near_plane       = 0.05f;
    s.camera.far_plane        = 100.0f;
    s.environment             = glm::vec3(0.05f, 0.06f, 0.08f);
    s.environment_texture     = texture(8, 4, 1.0f);
    s.environment_strength    = 0.75f;
    s.environment_rotation_degrees = 30.0f;

    const auto up = quad(false), down = quad(true);
    const auto checker = texture(4, 4, 0.0f), bumps = texture(2, 2, 0.5f);

    minirender::RenderInstance floor;
    floor.mesh                        = up;
    floor.material.kind               = minirender::MaterialKind::diffuse;
    floor.material.base_color         = glm::vec3(0.9f, 0.8f, 0.7f);
    floor.material.texture_filter     = minirender::TextureFilter::bilinear;
    floor.material.normal_scale       = 0.6f;
    floor.material.double_sided       = true;
    floor.object_to_world             = translate_scale({0, 0, 0}, {3, 1, 3});
    floor.normal_to_world             = inverse_scale({3, 1, 3});
    floor.base_color_texture          = checker;
    floor.normal_texture              = bumps;
    s.instances.push_back(floor);

    minirender::RenderInstance plate;
    plate.mesh                = up;
    plate.material.kind       = minirender::MaterialKind::conductor;
    plate.material.base_color = glm::vec3(0.95f, 0.7f, 0.4f);
    plate.material.roughness  = 0.3f;
    plate.object_to_world     = translate_scale({0.5f, 0.4f, -0.5f}, {0.5f, 1.0f, 0.25f});
    plate.normal_to_world     = inverse_scale({0.5f, 1.0f, 0.25f});
    s.instances.push_back(plate);

    minirender::RenderInstance light;
    light.mesh                  = down;
    light.material.kind         = minirender::MaterialKind::diffuse;
    light.material.base_color   = glm::vec3(0.0f);
    light.material.emission     = glm::vec3(6.0f, 5.0f, 4.0f);
    light.material.double_sided = false;
    light.object_to_world       = translate_scale({-0.5f, 2.0f, 0.5f}, {0.4f, 1.0f, 0.4f});
    light.normal_to_world       = inverse_scale({0.4f, 1.0f, 0.4f});
    s.instances.push_back(light);

    minirender::DirectionalLight sun;
    sun.direction = glm::vec3(-1.0f, -3.0f, -0.5f);
    sun.color     = glm::vec3(1.0f, 0.9f, 0.8f);
    sun.intensity = 2.0f;
    s.directional_lights.push_back(sun);

    minirender::MediumRegion fog;
    fog.minimum                  = glm::dvec3(-2.0, 0.0, -2.0);
    fog.maximum                  = glm::dvec3(2.0, 1.5, 2.0);
    fog.medium.absorption        = glm::dvec3(0.02, 0.03, 0.04);
    fog.medium.scattering        = glm::dvec3(0.1, 0.1, 0.1);
    fog.medium.anisotropy        = 0.3;
    s.media.push_back(fog);

    const B200Snapshot flat = to_b200(s);
    // The conversion shares the mesh and each texture once.
    if (flat.desc.mesh_count != 2 || flat.desc.instance_count != 3 || flat.desc.texture_count != 3 ||
        flat.desc.environment_texture != 3 || flat.desc.materials[0].base_color_texture != 1 ||
        flat.desc.materials[0].normal_texture != 2 || flat.desc.materials[1].base_color_texture != 0) {
        std::fprintf(stderr, "unexpected conversion: meshes %u instances %u textures %u env %u\n",
                     flat.desc.mesh_count, flat.desc.instance_count, flat.desc.texture_count,
                     flat.desc.environment_texture);
        return 1;
    }

    const mr_integrator_settings integrator{MR_SAMPLING_MIS, 5, 1, 3};
    const mr_render_settings     render{24, 16, 4, 7};
    void*                        scene = nullptr;
    char                         message[512];
    if (or_scene_create(&flat.desc, nullptr, &integrator, &scene) != 0) {
        or_last_error(message, sizeof(message));
        std::fprintf(stderr, "oracle refused the converted snapshot: %s\n", message);
        return 1;
    }
    std::vector<float> rgb(render.width * render.height * 3);
    mr_path_statistics stats{};
    const int          status = or_render_rows(scene, &render, 0, render.height, 1, rgb.data(), &stats);
    or_scene_destroy(scene);
    if (status != 0) {
        or_last_error(message, sizeof(message));
        std::fprintf(stderr, "oracle render failed: %s\n", message);
        return 1;
    }
    std::FILE* f = std::fopen(argv[1], "wb");
    if (!f || std::fwrite(rgb.data(), sizeof(float), rgb.size(), f) != rgb.size()) {
        return 1;
    }
    std::fclose(f);
    std::printf("converted and rendered: %u instances, %u textures\n", flat.desc.instance_count,
                flat.desc.texture_count);
    return 0;
}
