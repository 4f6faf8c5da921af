// Initial configurations (seeded diameters + RSA placement), host code.
#pragma once

#include <cstddef>
#include <cstdint>
#include <random>
#include <string>
#include <vector>

namespace rcpg {

// Distribution (initialize_particles.hpp:18-31).
struct DistSpec {
    std::string type = "mono";
    double d = 1.0;
    double mu = 1.0, sigma = 0.2;
    double mu1 = 1.0, sigma1 = 0.2;
    double mu2 = 2.0, sigma2 = 0.3;
    double p = 0.5;
    double d1 = 1.0, d2 = 2.0;
    double d_min = 0.5, d_max = 1.5;
    double exponent = -2.5;
    double scale = 1.0, shape = 2.0;
    std::vector<double> custom;
};

// InitializerConfig (initialize_particles.hpp:33-42).
struct InitSpec {
    double phi = 0.05;
    std::size_t N = 0;
    std::size_t ndim = 0;
    std::vector<double> box;
    std::vector<std::int8_t> walls;
    bool fix_height = false;
    DistSpec dist;
    std::uint64_t seed = 0;
};

// InitializerResult (initialize_particles.hpp:44-51).
struct InitResult {
    std::vector<double> positions;  // [N*ndim]
    std::vector<double> diameters;
    std::vector<double> box;
    std::vector<std::int8_t> walls;
    double scale_factor = 1.0;
    double phi_modifier = 1.0;
};

std::vector<double> draw_diameters(std::size_t N, const DistSpec& dist, std::mt19937& rng);
void place_rsa(std::vector<double>& x, const std::vector<double>& D, const std::vector<double>& box,
               const std::vector<std::int8_t>& walls, std::uint64_t seed);
InitResult initialize_particles(const InitSpec& spec);

}  // namespace rcpg
