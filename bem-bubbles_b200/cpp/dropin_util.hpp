// Helpers shared by the drop-in's translation units: vertex lists <-> flat double arrays of the C ABI.
#ifndef BEM_DROPIN_UTIL_HPP
#define BEM_DROPIN_UTIL_HPP

#include <vector>

#include "Bem/basic/Bem.hpp"

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

}  // namespace dropin
}  // namespace Bem

#endif  // BEM_DROPIN_UTIL_HPP
