// Render harness around the reference's own C API: TEST INFRASTRUCTURE, not product.
//
// Replays a recorded sequence of su_* calls (source/capi/sprout.h) against the reference
// library, statically linked (oracle/Makefile), renders, and writes the framebuffer.  The
// reference runs in its own process because its statically linked C++ runtime does not mix
// with the one a Python process has already loaded.
//
// usage: ref_render SCRIPT DATA OUT
//   SCRIPT: one command per line
//     init <progressive 0|1>
//     camera <width> <height> <fov radians>
//     trafo <handle> <16 floats, row-major object-to-world>
//     integrators <json>
//     sampler <spp>
//     defaults
//     material <json>
//     image <pixel type> <channels> <width> <height> <depth> <byte offset of the pixels>
//       (su_create_image, tightly packed; the created image id must equal the number of images
//       created before it, which the recorded material JSON refers to)
//     mesh <num_triangles> <num_vertices> <byte offset of positions> <of normals> <of indices>
//          [<num parts> <byte offset of the parts: (first index, index count, material slot)>
//           [<byte offset of the texture coordinates, 2 floats per vertex>]]
//     prop <mesh handle or built-in shape id (< 8)> <num materials> <material handles...>
//     light <prop handle>
//     mount <folder>   (su_mount; the folder name without spaces)
//     take <width> <height> <take file>   (su_load_take; the take's resolution, for the readback)
//     progressive <iterations>
//     prepare   (su_start_render_frame(0), timed apart as prepare_s: joins the asynchronous mesh
//               BVH builds and compiles the scene, so that a later "frame" times the render)
//     frame <frame>
//   Handles: the n-th camera/material/mesh/prop command creates handle 4000/1000+n/2000+n/3000+n.
//   DATA: raw little-endian arrays referenced by byte offset.
//   OUT: float32 RGBA framebuffer (width * height * 4).
// Prints one JSON line: render and preparation seconds and the su_* status codes.
#include "capi/sprout.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: ref_render SCRIPT DATA OUT\n");
        return 2;
    }
    FILE* df = std::fopen(argv[2], "rb");
    if (!df) {
        return 2;
    }
    std::fseek(df, 0, SEEK_END);
    long const dsize = std::ftell(df);
    std::fseek(df, 0, SEEK_SET);
    std::vector<char> data(size_t(dsize) + 16);
    if (dsize > 0 && 1 != std::fread(data.data(), size_t(dsize), 1, df)) {
        return 2;
    }
    std::fclose(df);

    FILE* sf = std::fopen(argv[1], "r");
    if (!sf) {
        return 2;
    }

    std::map<uint32_t, uint32_t> handles;
    uint32_t n_mat = 0, n_mesh = 0, n_prop = 0, n_image = 0;
    uint32_t width = 0, height = 0;
    double   render_s = 0.0;
    double   prepare_s = 0.0;
    int32_t  status   = 0;

    char line[1 << 16];
    while (std::fgets(line, sizeof(line), sf)) {
        char cmd[32] = {};
        int  used    = 0;
        if (std::sscanf(line, "%31s%n", cmd, &used) != 1) {
            continue;
        }
        char const*       rest = line + used;
        std::string const c(cmd);
        if (c == "init") {
            int p = 0;
            std::sscanf(rest, "%d", &p);
            status |= su_init(p != 0);
            // the reference's warnings and errors go to stderr
            su_register_log([](uint32_t type, char const* text) {
                if (type == SU_LOG_WARNING || type == SU_LOG_ERROR) {
                    std::fprintf(stderr, "reference log %u: %s\n", type, text);
                }
            });
        } else if (c == "camera") {
            float fov = 0.f;
            std::sscanf(rest, "%u %u %f", &width, &height, &fov);
            handles[4000] = su_create_camera_perspective(width, height, fov);
        } else if (c == "trafo") {
            uint32_t h = 0;
            float    m[16];
            std::sscanf(rest, "%u %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f %f", &h, &m[0],
                        &m[1], &m[2], &m[3], &m[4], &m[5], &m[6], &m[7], &m[8], &m[9], &m[10],
                        &m[11], &m[12], &m[13], &m[14], &m[15]);
            status |= su_entity_set_transformation(handles[h], m);
        } else if (c == "mount") {
            char folder[4096] = {};
            std::sscanf(rest, " %4095s", folder);
            status |= su_mount(folder);
        } else if (c == "take") {
            char path[4096] = {};
            std::sscanf(rest, "%u %u %4095s", &width, &height, path);
            status |= su_load_take(path);
        } else if (c == "integrators") {
            su_create_integrators(rest);
        } else if (c == "sampler") {
            uint32_t spp = 1;
            std::sscanf(rest, "%u", &spp);
            status |= su_create_sampler(spp);
        } else if (c == "defaults") {
            status |= su_create_defaults();
        } else if (c == "material") {
            handles[1000 + n_mat++] = su_create_material(rest);
        } else if (c == "image") {
            uint32_t type = 0, channels = 0, w = 0, h = 0, d = 0;
            size_t   off  = 0;
            std::sscanf(rest, "%u %u %u %u %u %zu", &type, &channels, &w, &h, &d, &off);
            uint32_t const bytes = type == 0 ? 1u : (type == 1 ? 2u : 4u);
            uint32_t const id    = su_create_image(type, channels, w, h, d, 0, bytes * channels,
                                                   data.data() + off);
            if (id != n_image++) {
                status |= 0x100;
            }
        } else if (c == "mesh") {
            uint32_t nt = 0, nv = 0, np = 0;
            size_t   op = 0, on = 0, oi = 0, opart = 0, ouv = 0;
            int const fields = std::sscanf(rest, "%u %u %zu %zu %zu %u %zu %zu", &nt, &nv, &op, &on, &oi, &np,
                                           &opart, &ouv);
            auto const* pos = reinterpret_cast<float const*>(data.data() + op);
            auto const* nrm = reinterpret_cast<float const*>(data.data() + on);
            auto const* idx = reinterpret_cast<uint32_t const*>(data.data() + oi);
            auto const* prt = np ? reinterpret_cast<uint32_t const*>(data.data() + opart) : nullptr;
            auto const* uvs = fields == 8 ? reinterpret_cast<float const*>(data.data() + ouv) : nullptr;
            handles[2000 + n_mesh++] = su_create_triangle_mesh_async(
                nt, nv, 3, pos, 3, nrm, 0, nullptr, uvs ? 2 : 0, uvs, idx, np, prt);
        } else if (c == "prop") {
            uint32_t mesh = 0, nm = 0;
            int      off  = 0;
            std::sscanf(rest, "%u %u%n", &mesh, &nm, &off);
            std::vector<uint32_t> mats(nm);
            char const*           p = rest + off;
            for (uint32_t i = 0; i < nm; ++i) {
                uint32_t h = 0;
                int      k = 0;
                std::sscanf(p, "%u%n", &h, &k);
                p += k;
                mats[i] = handles[h];
            }
            // ids below 8 are the built-in shapes (sprout.h:22-29), passed as they are
            uint32_t const shape = mesh < 8 ? mesh : handles[mesh];
            handles[3000 + n_prop++] = su_create_prop(shape, nm, mats.data());
        } else if (c == "light") {
            uint32_t h = 0;
            std::sscanf(rest, "%u", &h);
            status |= su_create_light(handles[h]);
        } else if (c == "progressive") {
            uint32_t it = 0;
            std::sscanf(rest, "%u", &it);
            auto const t0 = std::chrono::steady_clock::now();
            status |= su_start_render_frame(0);
            for (uint32_t i = 0; i < it; ++i) {
                status |= su_render_iteration();
            }
            render_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        } else if (c == "prepare") {
            auto const t0 = std::chrono::steady_clock::now();
            status |= su_start_render_frame(0);
            prepare_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        } else if (c == "frame") {
            uint32_t f = 0;
            std::sscanf(rest, "%u", &f);
            auto const t0 = std::chrono::steady_clock::now();
            status |= su_render_frame(f);
            render_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
    }
    std::fclose(sf);

    status |= su_postprocess();
    std::vector<float> fb(size_t(width) * height * 4, 0.f);
    // the reference copies and then returns -2 for SU_FLOAT32 (capi.cpp:704-714)
    su_copy_framebuffer(SU_FLOAT32, width, height, 4, reinterpret_cast<uint8_t*>(fb.data()));
    FILE* of = std::fopen(argv[3], "wb");
    if (!of) {
        return 2;
    }
    std::fwrite(fb.data(), sizeof(float), fb.size(), of);
    std::fclose(of);
    su_release();
    std::printf("{\"render_s\": %.6f, \"prepare_s\": %.6f, \"status\": %d}\n", render_s, prepare_s,
                status);
    return 0;
}
