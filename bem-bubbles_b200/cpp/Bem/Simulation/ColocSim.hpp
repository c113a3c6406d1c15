// Drop-in replacement of the reference's Bem::ColocSim (Bem/Simulation/ColocSim.hpp:13-28): collocation
// BEM with linear elements whose matrix assembly runs on the GPU.
#ifndef COLOCSIM_HPP
#define COLOCSIM_HPP

#include <iostream>
#include <vector>

#include "LinLinSim.hpp"

#include <Eigen/Dense>

namespace Bem {

class ColocSim : public LinLinSim {
public:
    ColocSim(Mesh const& initial, real p_inf = 1.0, real epsilon = 1.0, real sigma = 0.0, real gamma = 1.0,
             real (*pressurefield)(vec3 x, real t) = &default_field)
        : LinLinSim(initial, p_inf, epsilon, sigma, gamma, pressurefield) {}

    virtual ~ColocSim() {}

    // G and H of the collocation method for mesh m (ColocSim.cpp:21-110), assembled on the GPU
    virtual void assemble_matrices(Eigen::MatrixXd& G, Eigen::MatrixXd& H, Mesh const& m) const override;
};

}  // namespace Bem

#endif  // COLOCSIM_HPP
