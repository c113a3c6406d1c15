// Check of the drop-in's remesh projection (test infrastructure): the user's library function
// project_and_interpolate (Bem/Mesh/MeshManip.cpp:1416-1697, both overloads) against the drop-in's
// dropin::project_interpolate (ray casting on the GPU) on the same meshes, compared bit for bit, with
// the wall-clock time of each.  The new mesh is a perturbed sphere after the topology edits of a remesh;
// the old one is the perturbed sphere.  Usage: project_check <in.ply> <L>.  Exit status 0 when identical.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "Bem/Mesh/HalfedgeMesh.hpp"
#include "Bem/Mesh/MeshIO.hpp"
#include "Bem/Mesh/MeshManip.hpp"
#include "dropin_util.hpp"
#include "bem_b200.h"

using namespace Bem;
using clk = std::chrono::steady_clock;

static double ms_since(clk::time_point t0) {
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

int main(int argc, char* argv[]) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: project_check <in.ply> <L>\n");
        return 2;
    }
    Mesh old;
    import_ply(argv[1], old);
    const double L = std::atof(argv[2]);
    for (vec3& v : old.verts) v = v * (1.0 + 0.05 * std::sin(3.0 * v.z + v.y) * std::cos(2.0 * v.x));
    old.translate(vec3(3.0, 0.0, 0.0));
    std::vector<real> f(old.verts.size()), g(old.verts.size());
    for (size_t i = 0; i < f.size(); ++i) {
        f[i] = std::sin(old.verts[i].x) + 0.3 * old.verts[i].y;
        g[i] = std::cos(2.0 * old.verts[i].z);
    }
    // the topology edits of a remesh with a uniform density
    HalfedgeMesh he(generate_halfedges(old));
    std::vector<real> dens(old.verts.size(), 1.0);
    split_edges(he, dens, L * 0.75);
    flip_edges(he, 1);
    relax_vertices(he);
    collapse_edges(he, dens, L * 0.8);
    flip_edges(he, 1);
    relax_vertices(he);
    const Mesh next = generate_mesh(he);
    const CoordVec normals = generate_vertex_normals(next);

    bem_ctx* c = nullptr;
    if (bem_create(&c, 0, nullptr) != BEM_OK) {
        std::fprintf(stderr, "no CUDA device\n");
        return 2;
    }
    int bad = 0;
    for (int fitted = 1; fitted >= 0; --fitted) {
        Mesh a = next, b = next;
        std::vector<real> fa, fb, ga, gb;
        auto t0 = clk::now();
        if (fitted)
            project_and_interpolate(a, normals, fa, old, f);
        else
            project_and_interpolate(a, normals, fa, ga, old, f, g);
        const double t_lib = ms_since(t0);
        t0 = clk::now();
        dropin::project_interpolate(c, b, normals, old, f, fb, fitted ? nullptr : &g, fitted ? nullptr : &gb, fitted);
        const double t_gpu = ms_since(t0);
        size_t diff = 0;
        for (size_t i = 0; i < a.verts.size(); ++i) {
            diff += !(a.verts[i].x == b.verts[i].x && a.verts[i].y == b.verts[i].y && a.verts[i].z == b.verts[i].z);
            diff += !(fa[i] == fb[i]);
            if (!fitted) diff += !(ga[i] == gb[i]);
        }
        std::printf("project fitted %d new %zu old %zu trigs %zu differing %zu library_ms %.1f dropin_ms %.1f\n", fitted,
                    next.verts.size(), old.verts.size(), old.trigs.size(), diff, t_lib, t_gpu);
        bad += diff != 0;
    }
    bem_destroy(c);
    return bad ? 1 : 0;
}
