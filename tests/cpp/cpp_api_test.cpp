// Drives the C++ mirror classes (include/cpt.hpp) the way the reference application
// drives CUDA::BVHBuilder and CUDAPathTracer, and writes what they produced for
// tests/test_gpu_cpp_api.py to compare with the oracle and the C ABI path.
//   usage: cpp_api_test <output dir>
#include <cstdio>
#include <string>
#include <vector>
#include "cpt.hpp"

namespace {

template <typename T>
bool write(const std::string& path, const std::vector<T>& v)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t n = std::fwrite(v.data(), sizeof(T), v.size(), f);
    std::fclose(f);
    return n == v.size();
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <output dir>\n", argv[0]);
        return 2;
    }
    const std::string out = argv[1];
    const uint32_t n_random = 20000;
    cpt::HostSceneDescription scene;
    scene.triangles.resize(n_random + 2);
    scene.triangleInfo.resize(n_random + 2);
    const uint32_t n = cpt_scene_random(n_random, 4, 0.005f, 0.02f, 0.7f, 1.25f, 0.5f, 10.0f, scene.triangles.data(),
                                        scene.triangleInfo.data());
    scene.triangles.resize(n);
    scene.triangleInfo.resize(n);
    float box[6];
    cpt_scene_bounds(scene.triangles.data(), n, box);
    for (int a = 0; a < 3; ++a) {
        scene.enclosingBBox.min[a] = box[a];
        scene.enclosingBBox.max[a] = box[3 + a];
    }

    // Scene::upload's build step (Scene.cu:28-55)
    cpt::DeviceSceneDescription desc;
    desc.triangles.assign(scene.triangles.data(), n);
    desc.enclosingBBox = scene.enclosingBBox;
    cpt::BVHBuilder<30> builder;
    builder.build(desc, n);
    if (cpt::last_error() != CPT_OK) return 1;
    if (!write(out + "/tris.bin", desc.triangles.to_host()) || !write(out + "/children.bin", desc.children.to_host()) ||
        !write(out + "/parents_leaf.bin", desc.parents[cpt::LEAF_PARENTS_IDX].to_host()) ||
        !write(out + "/parents_internal.bin", desc.parents[cpt::INTERNAL_PARENTS_IDX].to_host()) ||
        !write(out + "/boxes.bin", desc.internalNodeBBoxes.to_host()))
        return 1;

    // PathTracingApp's per-frame calls (PathTracingApp.cpp:269-285)
    cpt::CUDAPathTracer tracer(30);
    tracer.setSettings(3, 3.0f, true, 7);
    tracer.upload(scene);
    cpt_camera cam{};
    const float eye[3] = {0.5f, 0.5f, -1.2f}, target[3] = {0.5f, 0.5f, 0.0f}, up[3] = {0.0f, 1.0f, 0.0f};
    cpt_camera_look_at(eye, target, up, 45.0f, 48.0f / 32.0f, 0.3f, 30.0f, &cam);
    auto ray = [&](int c) {
        return cpt::Ray{{cam.eye[0], cam.eye[1], cam.eye[2]}, {cam.dirs[c][0], cam.dirs[c][1], cam.dirs[c][2]}};
    };
    tracer.setPrimaryRays(ray(0), ray(1), ray(2), ray(3));
    tracer.setEyePos({cam.eye[0], cam.eye[1], cam.eye[2]});
    tracer.raytrace(48, 32);
    tracer.raytrace(48, 32);
    if (cpt::last_error() != CPT_OK) return 1;
    if (!write(out + "/image.bin", tracer.readImage(48, 32))) return 1;
    std::printf("frames %u\n", tracer.frame());

    // the extensions: split and wide traversal trees, next-event estimation
    cpt::CUDAPathTracer fast(30);
    fast.setSettings(3, 3.0f, true, 7);
    fast.setSplit(2.0f);
    fast.setWide(true);
    fast.setNextEventEstimation(true);
    fast.upload(scene);
    fast.setPrimaryRays(ray(0), ray(1), ray(2), ray(3));
    fast.setEyePos({cam.eye[0], cam.eye[1], cam.eye[2]});
    fast.raytrace(48, 32);
    if (cpt::last_error() != CPT_OK) return 1;
    if (!write(out + "/image_ext.bin", fast.readImage(48, 32))) return 1;

    // error behaviour: reported and kept, the tracer stays usable
    tracer.raytrace(0, 32);
    if (cpt::last_error() != CPT_ERR_INVALID_ARGUMENT) return 1;
    cpt::last_error() = CPT_OK;
    cpt::error_policy() = cpt::OnError::Throw;
    bool threw = false;
    try {
        tracer.raytrace(-1, 32);
    } catch (const std::runtime_error&) {
        threw = true;
    }
    if (!threw) return 1;
    std::printf("cpp api ok\n");
    return 0;
}
