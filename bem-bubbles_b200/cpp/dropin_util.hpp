// Helpers shared by the drop-in's translation units: vertex lists <-> flat double arrays of the C ABI.
#ifndef BEM_DROPIN_UTIL_HPP
#define BEM_DROPIN_UTIL_HPP

#include <vector>

#include "Bem/basic/Bem.hpp"
#include "Bem/Mesh/Mesh.hpp"

struct bem_ctx;

namespace Bem {
namespace dropin {

inline std::vector<double> flat(std::vector<vec3> const& v) {
    std::vector<double> out(3 * v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
    return out;
}

inline std::vector<vec3> unflat(std::vector<double> const& f) {
    std::vector<vec3> out(f.size() / 3);
    for (size_t i = 0; i < out.size(); ++i) out[i] = vec3(f[3 * i], f[3 * i + 1], f[3 * i + 2]);
    return out;
}

// project_and_interpolate (Bem/Mesh/MeshManip.cpp:1426-1697) with the ray casting on the device of
// context c: the vertices of `mesh` move along `normals` onto `other`; f (and f2) are interpolated
// linearly on the triangle hit.  fitted: the hit point is lifted onto the quadratic fits of the old
// surface (the one-function overload, :1426-1559); otherwise it stays on the flat triangle (the
// two-function overload, :1561-1697, whose fits the reference computes but does not use).
void project_interpolate(bem_ctx* c, Mesh& mesh, CoordVec const& normals, Mesh const& other,
                         std::vector<real> const& f, std::vector<real>& f_res, std::vector<real> const* f2,
                         std::vector<real>* f2_res, bool fitted);

}  // namespace dropin
}  // namespace Bem

#endif  // BEM_DROPIN_UTIL_HPP
