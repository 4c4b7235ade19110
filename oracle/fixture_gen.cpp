// Oracle (test infrastructure only): CPU restatement of the reference's
// seeded fixture generator, so that the reference's golden files
// (tests/data/n{N}_b{B}_s{seed}_{random,nearid}.bin) can be regenerated
// bit-for-bit from (N, B, seed, mode) without shipping their 31 MB of inputs.
//
// Follows tests/common/lapack_reference.cpp of the reference:
//   * one std::mt19937_64 seeded with `seed` drives the whole batch (:171)
//   * per matrix, H first, then S (:174-181)
//   * H = A + A^H with A(i,j) = N(0,1) + i N(0,1), drawn column-major
//     (:86-101). The reference writes `cdouble(g(rng), g(rng))`; GCC
//     evaluates those two arguments right to left, so the IMAGINARY part is
//     the first draw. Checked: with this order all 15 reference fixtures
//     regenerate bit-for-bit.
//   * random S    = A A^H + N I, A drawn the same way (:105-127)
//   * near-id S   = (1 + N/2) I + 0.1 (B + B^H) (:132-150)
// Draws come from std::normal_distribution<double>(0, 1), constructed fresh
// for every matrix as the reference does; with libstdc++ that is the
// Marsaglia polar method over std::generate_canonical, which is what makes
// the stream reproducible here (the fixtures were made with libstdc++).
//
// Output layout: column-major N x N per matrix, batch-contiguous
// (element (i, j) of matrix b at b*N*N + j*N + i), interleaved re/im doubles.
//
// Built by build() in oracle/fixtures.py into oracle/_build/libgeig_fixture.so
// and loaded with ctypes by the tests only.

#include <complex>
#include <cstdint>
#include <random>
#include <vector>

namespace {

using cd = std::complex<double>;

void draw_gaussian_matrix(int n, std::mt19937_64& rng, std::vector<cd>& A) {
    std::normal_distribution<double> nd(0.0, 1.0);
    A.assign(static_cast<size_t>(n) * n, cd(0.0, 0.0));
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            const double im = nd(rng);
            const double re = nd(rng);
            A[static_cast<size_t>(j) * n + i] = cd(re, im);
        }
}

void hermitian_from_gaussian(int n, std::mt19937_64& rng, cd* out) {
    std::vector<cd> A;
    draw_gaussian_matrix(n, rng, A);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            out[static_cast<size_t>(j) * n + i] =
                A[static_cast<size_t>(j) * n + i] + std::conj(A[static_cast<size_t>(i) * n + j]);
}

void spd_wide(int n, std::mt19937_64& rng, cd* out) {
    std::vector<cd> A;
    draw_gaussian_matrix(n, rng, A);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            cd acc(0.0, 0.0);
            for (int k = 0; k < n; ++k)
                acc += A[static_cast<size_t>(k) * n + i] * std::conj(A[static_cast<size_t>(k) * n + j]);
            out[static_cast<size_t>(j) * n + i] = acc;
        }
    for (int i = 0; i < n; ++i) out[static_cast<size_t>(i) * n + i] += cd(static_cast<double>(n), 0.0);
}

void spd_near_identity(int n, std::mt19937_64& rng, cd* out) {
    std::vector<cd> Bm;
    draw_gaussian_matrix(n, rng, Bm);
    const double shift = 1.0 + 0.5 * static_cast<double>(n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            cd v = 0.1 * (Bm[static_cast<size_t>(j) * n + i] + std::conj(Bm[static_cast<size_t>(i) * n + j]));
            if (i == j) v += cd(shift, 0.0);
            out[static_cast<size_t>(j) * n + i] = v;
        }
}

}  // namespace

extern "C" {

// mode 0 = random wide-spectrum S, mode 1 = near-identity S.
// H_out, S_out: n*n*batch complex (2 doubles each). Returns 0 on success.
int geig_fixture_generate(int n, int batch, long long seed, int mode, double* H_out, double* S_out) {
    if (n <= 0 || batch < 0 || !H_out || !S_out || (mode != 0 && mode != 1)) return -1;
    std::mt19937_64 rng(static_cast<std::uint64_t>(seed));
    const size_t mat = static_cast<size_t>(n) * n;
    cd* H = reinterpret_cast<cd*>(H_out);
    cd* S = reinterpret_cast<cd*>(S_out);
    for (int b = 0; b < batch; ++b) {
        hermitian_from_gaussian(n, rng, H + mat * b);
        if (mode == 0) spd_wide(n, rng, S + mat * b);
        else           spd_near_identity(n, rng, S + mat * b);
    }
    return 0;
}

}  // extern "C"
