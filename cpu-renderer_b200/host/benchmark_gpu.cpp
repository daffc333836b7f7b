// GPU drop-in for CPU-Renderer's manual phase benchmark (tests/benchmark.cpp): the same
// command line (scene.glb sky.hdr), the same scene loading (the reference's io::loadGltf,
// Bvh::build and Environment), the same seven phases over 400,000 calls and the same report
// lines, with every phase run as one kernel on the GPU (cr_gpu_phase_benchmark) and timed
// with CUDA events. Camera rays are the reference's (see cr_gpu_phase_benchmark); the BSDF and
// environment phases draw each call from its own stream, so their checksum terms differ from
// the CPU run's while the hit count and the traversal terms match it.
#include "render.h"
#include "render_gpu.h"

#include <cmath>
#include <cstring>
#include <iomanip>
#include <iostream>

using namespace cr;

int main(int argc, char** argv) {
    try {
        if (argc != 3) throw std::runtime_error("Usage: renderer_benchmark scene.glb sky.hdr");
        Scene scene = io::loadGltf(argv[1]);
        if (scene.cameras.empty()) throw std::runtime_error("Benchmark scene needs a camera");
        Bvh bvh;
        bvh.build(scene);
        Environment sky(io::loadImage(argv[2], true), 0, 1);
        cr_gpu_scene* g = uploadToGpu(scene, bvh, sky, 0);
        const Camera& camera = scene.cameras[0];
        cr_camera c{};
        std::memcpy(c.position, &camera.position, 12);
        std::memcpy(c.forward, &camera.forward, 12);
        std::memcpy(c.right, &camera.right, 12);
        std::memcpy(c.up, &camera.up, 12);
        c.yfov = camera.yfov; c.aspect = camera.aspect; c.near_clip = camera.nearClip; c.far_clip = camera.farClip;
        constexpr uint32_t count = 400000;
        cr_phase_timing t[CR_PHASE_COUNT];
        const cr_status st = cr_gpu_phase_benchmark(g, &c, 320, 180, count, 42, t);
        if (st != CR_OK) {
            char buf[1024];
            cr_gpu_last_error(buf, sizeof(buf));
            cr_gpu_scene_destroy(g);
            throw std::runtime_error(buf);
        }
        const char* names[CR_PHASE_COUNT] = {"camera", "closest-hit traversal", "occlusion traversal", "surface shading/maps",
                                             "BSDF sampling", "BSDF evaluation", "HDR importance sample+lookup+PDF"};
        double checksum = 0;
        for (int k = 0; k < CR_PHASE_COUNT; ++k) {
            std::cout << std::fixed << std::setprecision(3) << names[k] << ": " << t[k].seconds << " s, "
                      << t[k].seconds * 1e9 / static_cast<double>(t[k].calls ? t[k].calls : 1) << " ns/call, " << t[k].calls
                      << " calls\n";
            checksum += t[k].checksum;
        }
        std::cout << "triangles=" << scene.triangles.size() << " hits=" << t[CR_PHASE_SURFACE].calls << " checksum=" << checksum
                  << '\n';
        cr_gpu_scene_destroy(g);
        return std::isfinite(checksum) ? 0 : 1;
    } catch (const std::exception& error) {
        std::cerr << error.what() << '\n';
        return 1;
    }
}
