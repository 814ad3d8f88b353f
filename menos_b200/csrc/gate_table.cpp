// Gate matrices for the named gates, bit for bit the reference's
// ir::generate_matrix (src/ir/gate_table.cpp:17-206, :260).  The same
// expressions, evaluated by the same libstdc++/glibc (std::exp of a
// std::complex<double> is glibc's cexp; std::cos/std::sin are libm's), built
// with -ffp-contract=off, give the same bytes on the same host.  The
// expressions have to stay textually equivalent to the reference's; the
// oracle pin (tests/test_oracle_pin.py) checks every gate against it.
#include <cmath>
#include <complex>
#include <cstring>
#include <numbers>
#include <vector>

#include "mb2_internal.h"

namespace mb2 {
namespace {

using Cd = std::complex<double>;
using namespace std::complex_literals;
constexpr double kPi = std::numbers::pi_v<double>;

}  // namespace

int gate_num_qubits(int opcode) {
    if (opcode >= MB2_X && opcode <= MB2_U) return 1;
    if (opcode >= MB2_CX && opcode <= MB2_RZZ) return 2;
    if (opcode == MB2_CCX) return 3;
    return 0;
}

int gate_num_params(int opcode) {
    switch (opcode) {
        case MB2_RX: case MB2_RY: case MB2_RZ: case MB2_P: case MB2_CP: case MB2_RZZ: return 1;
        case MB2_U: return 3;
        default: return 0;
    }
}

// Fills `m` (row-major, dim*dim entries) and returns dim; 0 for an opcode
// that names no gate matrix.
int gate_matrix(int opcode, const double* params, std::vector<Cd>& m) {
    switch (opcode) {
        case MB2_X: m = {0.0, 1.0, 1.0, 0.0}; return 2;
        case MB2_Y: m = {0.0, -1.0i, 1.0i, 0.0}; return 2;
        case MB2_Z: m = {1.0, 0.0, 0.0, -1.0}; return 2;
        case MB2_H: {
            const double s = 1.0 / std::sqrt(2.0);
            m = {s, s, s, -s};
            return 2;
        }
        case MB2_S: m = {1.0, 0.0, 0.0, 1.0i}; return 2;
        case MB2_SDG: m = {1.0, 0.0, 0.0, -1.0i}; return 2;
        case MB2_T: m = {1.0, 0.0, 0.0, std::exp(1.0i * (kPi / 4.0))}; return 2;
        case MB2_TDG: m = {1.0, 0.0, 0.0, std::exp(-1.0i * (kPi / 4.0))}; return 2;
        case MB2_SX:
            m = {0.5 * (1.0 + 1.0i), 0.5 * (1.0 - 1.0i), 0.5 * (1.0 - 1.0i), 0.5 * (1.0 + 1.0i)};
            return 2;
        case MB2_SXDG:
            m = {0.5 * (1.0 - 1.0i), 0.5 * (1.0 + 1.0i), 0.5 * (1.0 + 1.0i), 0.5 * (1.0 - 1.0i)};
            return 2;
        case MB2_RX: {
            const double theta = params[0];
            const double c = std::cos(theta / 2.0);
            const double s = std::sin(theta / 2.0);
            m = {c, -1.0i * s, -1.0i * s, c};
            return 2;
        }
        case MB2_RY: {
            const double theta = params[0];
            const double c = std::cos(theta / 2.0);
            const double s = std::sin(theta / 2.0);
            m = {c, -s, s, c};
            return 2;
        }
        case MB2_RZ: {
            const double theta = params[0];
            m = {std::exp(-1.0i * (theta / 2.0)), 0.0, 0.0, std::exp(1.0i * (theta / 2.0))};
            return 2;
        }
        case MB2_P: {
            const double lambda = params[0];
            m = {1.0, 0.0, 0.0, std::exp(1.0i * lambda)};
            return 2;
        }
        case MB2_U: {
            const double theta = params[0];
            const double phi = params[1];
            const double lambda = params[2];
            const double c = std::cos(theta / 2.0);
            const double s = std::sin(theta / 2.0);
            m = {c, -std::exp(1.0i * lambda) * s, std::exp(1.0i * phi) * s,
                 std::exp(1.0i * (phi + lambda)) * c};
            return 2;
        }
        case MB2_CX:
            m.assign(16, 0.0);
            m[0] = 1.0; m[7] = 1.0; m[10] = 1.0; m[13] = 1.0;
            return 4;
        case MB2_CZ:
            m.assign(16, 0.0);
            m[0] = 1.0; m[5] = 1.0; m[10] = 1.0; m[15] = -1.0;
            return 4;
        case MB2_SWAP:
            m.assign(16, 0.0);
            m[0] = 1.0; m[6] = 1.0; m[9] = 1.0; m[15] = 1.0;
            return 4;
        case MB2_CP: {
            const double lambda = params[0];
            m.assign(16, 0.0);
            m[0] = 1.0; m[5] = 1.0; m[10] = 1.0;
            m[15] = std::exp(1.0i * lambda);
            return 4;
        }
        case MB2_RZZ: {
            const double theta = params[0];
            const Cd same = std::exp(-0.5i * theta);
            const Cd diff = std::exp(0.5i * theta);
            m.assign(16, 0.0);
            m[0] = same; m[5] = diff; m[10] = diff; m[15] = same;
            return 4;
        }
        case MB2_CCX:
            m.assign(64, 0.0);
            for (int i = 0; i < 8; ++i) m[i * 8 + i] = 1.0;
            m[3 * 8 + 3] = 0.0;
            m[7 * 8 + 7] = 0.0;
            m[3 * 8 + 7] = 1.0;
            m[7 * 8 + 3] = 1.0;
            return 8;
        default:
            return 0;
    }
}

// exp(i * global_phase), as the reference's initialize computes it
// (src/kernels/cpu/dense_kernels.cpp:22).
Cd initial_phase(double global_phase) {
    return std::exp(std::complex<double>{0.0, global_phase});
}

}  // namespace mb2

extern "C" int mb2_gate_matrix(int32_t opcode, const double* params, double* out, uint32_t out_len) {
    std::vector<std::complex<double>> m;
    double zero[3] = {0.0, 0.0, 0.0};
    const int dim = mb2::gate_matrix(opcode, params != nullptr ? params : zero, m);
    if (dim == 0 || out == nullptr || out_len < 2u * dim * dim) return MB2_ERR_INVALID;
    std::memcpy(out, m.data(), m.size() * sizeof(std::complex<double>));
    return MB2_OK;
}
