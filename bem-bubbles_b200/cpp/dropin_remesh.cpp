// Projection step of the drop-in's remeshing: project_and_interpolate (Bem/Mesh/MeshManip.cpp:1426-1697)
// with its O(P x M) ray casting on the GPU (bem_trace_mesh).  The host keeps the O(N) parts with the
// user's mesh library: the quadratic surface fits around the old vertices (FittingTool), the local
// triangle coordinates and the linear interpolation of the surface values.  The arithmetic is the
// reference's, expression by expression, so the projected positions and interpolated values are
// bit-identical to the library function's; it runs single-threaded (the library version runs its
// loop on omp_set_num_threads(100) threads with per-thread copies of both meshes).
#include <cstdio>
#include <stdexcept>
#include <string>

#include "Bem/Mesh/FittingTool.hpp"
#include "Bem/Mesh/Mesh.hpp"
#include "../../include/bem_b200.h"
#include "dropin_util.hpp"

namespace Bem {
namespace dropin {

void project_interpolate(bem_ctx* c, Mesh& mesh, CoordVec const& normals, Mesh const& other,
                         std::vector<real> const& f, std::vector<real>& f_res, std::vector<real> const* f2,
                         std::vector<real>* f2_res, bool fitted) {
    const size_t n = mesh.verts.size();
    // rays from the new vertices along their normals onto the old surface
    std::vector<double> x = flat(other.verts), pos = flat(mesh.verts), dir = flat(normals);
    std::vector<int64_t> t(3 * other.trigs.size());
    for (size_t j = 0; j < other.trigs.size(); ++j)
        for (size_t k = 0; k < 3; ++k) t[3 * j + k] = (int64_t)other.trigs[j][k];
    std::vector<double> hit(3 * n);
    std::vector<int64_t> tri(n);
    std::vector<int32_t> ok(n);
    const int rc = bem_trace_mesh(c, (int64_t)other.verts.size(), x.data(), (int64_t)other.trigs.size(), t.data(),
                                  (int64_t)n, pos.data(), dir.data(), hit.data(), tri.data(), ok.data());
    if (rc != BEM_OK) throw std::runtime_error(std::string("remesh projection: ") + bem_last_error(c));
    // A ray that meets no old triangle leaves its vertex at the origin with triangle 0, as the
    // reference's project_and_interpolate does (it ignores trace_mesh's result); say so, since the
    // resulting mesh is degenerate and its solves slow or ill-posed.
    size_t missed = 0;
    for (size_t i = 0; i < n; ++i) missed += ok[i] ? 0 : 1;
    if (missed)
        std::fprintf(stderr, "remesh projection: %zu of %zu rays met no triangle of the old surface; those vertices "
                             "are placed at the origin, as the reference does\n", missed, n);

    // quadratic fits over each old vertex and its neighbours (MeshManip.cpp:1438-1448)
    std::vector<FittingTool> fits;
    if (fitted) {
        const std::vector<vec3> other_normals = generate_vertex_normals(other);
        const std::vector<std::vector<size_t>> nbr = generate_neighbours(other);
        fits.resize(other.verts.size());
        for (size_t i = 0; i < other.verts.size(); ++i) {
            std::vector<vec3> pts;
            pts.push_back(other.verts[i]);
            for (size_t j : nbr[i]) pts.push_back(other.verts[j]);
            fits[i].compute_quadratic_fit(other_normals[i], other.verts[i], pts);
        }
    }

    std::vector<vec3> moved(n);
    std::vector<real> res(n), res2(f2 ? n : 0);
    for (size_t i = 0; i < n; ++i) {
        vec3 p(hit[3 * i], hit[3 * i + 1], hit[3 * i + 2]);
        const Triplet tr = other.trigs[(size_t)tri[i]];
        const vec3 &A = other.verts[tr.a], &B = other.verts[tr.b], &C = other.verts[tr.c];
        vec3 Pa, Pb, Pc;
        if (fitted) {  // the hit point lifted onto each corner's fit (MeshManip.cpp:1486-1507)
            const FittingTool &fa = fits[tr.a], &fb = fits[tr.b], &fc = fits[tr.c];
            Pa = fa.copy_coord_system().transform(p);
            Pb = fb.copy_coord_system().transform(p);
            Pc = fc.copy_coord_system().transform(p);
            Pa = fa.get_position(Pa.x, Pa.y);
            Pb = fb.get_position(Pb.x, Pb.y);
            Pc = fc.get_position(Pc.x, Pc.y);
        }
        // coordinates (q, r) of the hit point in the old triangle's plane (MeshManip.cpp:1515-1539)
        vec3 u(B - A);
        u.normalize();
        vec3 v(C - B);
        v = v - v.dot(u) * u;
        v.normalize();
        const vec3 a(B - A), b(C - B), d(p - A);
        const real a0 = a.dot(u), a1 = a.dot(v), b0 = b.dot(u), b1 = b.dot(v), x0 = d.dot(u), x1 = d.dot(v);
        const real q = (x1 * b0 - b1 * x0) / (a1 * b0 - a0 * b1);
        const real r = (a1 * x0 - a0 * x1) / (a1 * b0 - a0 * b1);
        if (fitted) p = (1.0 - q) * Pa + (q - r) * Pb + r * Pc;
        moved[i] = p;
        res[i] = (1.0 - q) * f[tr.a] + (q - r) * f[tr.b] + r * f[tr.c];
        if (f2) res2[i] = (1.0 - q) * (*f2)[tr.a] + (q - r) * (*f2)[tr.b] + r * (*f2)[tr.c];
    }
    mesh.verts = moved;
    f_res = res;
    if (f2_res) *f2_res = res2;
}

}  // namespace dropin
}  // namespace Bem
