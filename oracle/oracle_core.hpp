// oracle_core.hpp — CPU restatement of the reference's ensemble SDE hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load it; the product (the CUDA library
// under stochasticphysics_b200/) never does.
//
// Parity status: the problem functions (deterministic vector, stochastic
// matrix, Ito->Stratonovich drift, Jacobians, rotation/finish logic) and the
// Neel parameter formulas are pinned by the reference's own Mathematica
// golden vectors (Tests/*, extracted by tests/golden/make_golden.py).  The
// solver step formulas, the window sampling, the ensemble mean, cubic
// anisotropy and the fields are restated from the cited source lines and are
// NOT pinned by any reference test (the reference cannot be built here:
// Eigen/MyCEL/SerAr/Boost are absent).  The Newton driver of ImplicitMidpoint
// lives in MyCEL (out of tree) and is restated from the in-file legacy loop:
// parity unpinned.
//
// Everything is templated on the scalar type T so the same code runs in
// double, long double and an operation-counting type (flop roofline).
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>

namespace orc {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 6.28318530717958647692;
// Boltzmann constant as written in Problems/Helpers/ParameterCalculatorNeel.h:43
constexpr double kB = 1.3806485279E-23;

// ---------------------------------------------------------------- small linear algebra
template <class T, int N>
struct Vec {
    T a[N];
    T& operator[](int i) { return a[i]; }
    const T& operator[](int i) const { return a[i]; }
    static Vec zero() {
        Vec v;
        for (int i = 0; i < N; ++i) v.a[i] = T(0.0);
        return v;
    }
};
template <class T, int R, int C>
struct Mat {
    T a[R][C];
    T& operator()(int r, int c) { return a[r][c]; }
    const T& operator()(int r, int c) const { return a[r][c]; }
    static Mat zero() {
        Mat m;
        for (int r = 0; r < R; ++r)
            for (int c = 0; c < C; ++c) m.a[r][c] = T(0.0);
        return m;
    }
    static Mat identity() {
        Mat m = zero();
        for (int r = 0; r < R && r < C; ++r) m.a[r][r] = T(1.0);
        return m;
    }
};
template <class T> using V3 = Vec<T, 3>;
template <class T> using M3 = Mat<T, 3, 3>;

template <class T, int N> Vec<T, N> operator+(const Vec<T, N>& x, const Vec<T, N>& y) {
    Vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = x[i] + y[i]; return r;
}
template <class T, int N> Vec<T, N> operator-(const Vec<T, N>& x, const Vec<T, N>& y) {
    Vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = x[i] - y[i]; return r;
}
template <class T, int N> Vec<T, N> operator*(const T& s, const Vec<T, N>& x) {
    Vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = s * x[i]; return r;
}
template <class T, int N> Vec<T, N> operator*(const Vec<T, N>& x, const T& s) {
    Vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = x[i] * s; return r;
}
template <class T, int N> T dot(const Vec<T, N>& x, const Vec<T, N>& y) {
    T s = x[0] * y[0]; for (int i = 1; i < N; ++i) s = s + x[i] * y[i]; return s;
}
template <class T> V3<T> cross(const V3<T>& x, const V3<T>& y) {
    V3<T> r;
    r[0] = x[1] * y[2] - x[2] * y[1];
    r[1] = x[2] * y[0] - x[0] * y[2];
    r[2] = x[0] * y[1] - x[1] * y[0];
    return r;
}
template <class T, int R, int C> Vec<T, R> operator*(const Mat<T, R, C>& m, const Vec<T, C>& v) {
    Vec<T, R> r;
    for (int i = 0; i < R; ++i) { T s = m(i, 0) * v[0]; for (int j = 1; j < C; ++j) s = s + m(i, j) * v[j]; r[i] = s; }
    return r;
}
template <class T, int R, int K, int C> Mat<T, R, C> operator*(const Mat<T, R, K>& a, const Mat<T, K, C>& b) {
    Mat<T, R, C> r;
    for (int i = 0; i < R; ++i)
        for (int j = 0; j < C; ++j) { T s = a(i, 0) * b(0, j); for (int k = 1; k < K; ++k) s = s + a(i, k) * b(k, j); r(i, j) = s; }
    return r;
}
template <class T, int R, int C> Mat<T, R, C> operator*(const T& s, const Mat<T, R, C>& m) {
    Mat<T, R, C> r; for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) r(i, j) = s * m(i, j); return r;
}
template <class T, int R, int C> Mat<T, R, C> operator*(const Mat<T, R, C>& m, const T& s) {
    Mat<T, R, C> r; for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) r(i, j) = m(i, j) * s; return r;
}
template <class T, int R, int C> Mat<T, R, C> operator+(const Mat<T, R, C>& x, const Mat<T, R, C>& y) {
    Mat<T, R, C> r; for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) r(i, j) = x(i, j) + y(i, j); return r;
}
template <class T, int R, int C> Mat<T, R, C> operator-(const Mat<T, R, C>& x, const Mat<T, R, C>& y) {
    Mat<T, R, C> r; for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) r(i, j) = x(i, j) - y(i, j); return r;
}
// outer product u v^T
template <class T> M3<T> outer(const V3<T>& u, const V3<T>& v) {
    M3<T> r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r(i, j) = u[i] * v[j]; return r;
}
// the cross-product matrix [v]x (so that [v]x w = v x w)
template <class T> M3<T> crossmat(const V3<T>& v) {
    M3<T> m = M3<T>::zero();
    m(0, 1) = -v[2]; m(0, 2) = v[1];
    m(1, 0) = v[2];  m(1, 2) = -v[0];
    m(2, 0) = -v[1]; m(2, 1) = v[0];
    return m;
}

// ---------------------------------------------------------------- parameters (always double)
// Problems/Helpers/ParameterCalculatorNeel.h:44-92
struct NeelParamsD {
    double NeelFactor1, NeelFactor2, DriftPrefactor, NoisePrefactor, Damping;
};
// V = 4/3 pi r^3 (MyCEL math::geometry::sphere::calcVolume, out of tree:
// MagneticProperties.h:159, HydrodynamicProperties.h:46)
inline double sphere_volume(double r) { return 4.0 / 3.0 * kPi * r * r * r; }

inline NeelParamsD calc_neel_params(double radius, double Ms, double alpha, double gamma, double temperature) {
    NeelParamsD p{};
    const double moment = sphere_volume(radius) * Ms;  // getSaturationMoment, MagneticProperties.h:166
    double diffsquare = 2.0 * alpha * kB * temperature / (gamma * moment);
    if (std::isinf(diffsquare) || std::isnan(diffsquare)) diffsquare = 0.0;
    if (std::isinf(alpha)) {
        p.NeelFactor1 = 0.0;
        p.NeelFactor2 = 0.0;
    } else {
        p.NeelFactor1 = -gamma / (1.0 + std::pow(alpha, 2));
        p.NeelFactor2 = std::abs(p.NeelFactor1) * alpha;
    }
    p.DriftPrefactor = (diffsquare == 0.0) ? 0.0 : -1.0 * std::pow(p.NeelFactor1, 2) * (1.0 + std::pow(alpha, 2)) * diffsquare;
    p.NoisePrefactor = std::sqrt(diffsquare);
    p.Damping = alpha;
    return p;
}

// Problems/Helpers/ParameterCalculatorBrown.h:39-58
struct BrownParamsD {
    double BrownPrefactor, BrownDiffusion, Brown_F_Noise;
};
inline BrownParamsD calc_brown_params(double rh, double viscosity, double temperature) {
    BrownParamsD p{};
    const double vh = sphere_volume(rh);
    p.BrownPrefactor = 1.0 / (6.0 * viscosity * vh);
    p.BrownDiffusion = std::sqrt(2.0 * kB * temperature * (6.0 * viscosity * vh));
    if (std::isinf(p.BrownDiffusion) || std::isnan(p.BrownDiffusion)) p.BrownDiffusion = 0.0;
    if (std::isnan(p.BrownPrefactor)) p.BrownPrefactor = 0.0;
    p.Brown_F_Noise = p.BrownPrefactor * p.BrownDiffusion;
    return p;
}

// Euler angles (phi, theta, psi) -> body axes in world coordinates.
// Problems/NeelRelaxation.h:240-260 and
// Problems/Helpers/ParticleStateInitializer.h:64-105 (identical formulas).
template <class T>
inline void euler_to_axes(const double e[3], V3<T>& x, V3<T>& y, V3<T>& z) {
    const double cphi = std::cos(e[0]), ctheta = std::cos(e[1]), cpsi = std::cos(e[2]);
    const double sphi = std::sin(e[0]), stheta = std::sin(e[1]), spsi = std::sin(e[2]);
    const double cphicpsi = cphi * cpsi, sphicpsi = sphi * cpsi, cphispsi = cphi * spsi, sphispsi = sphi * spsi;
    x[0] = T(cphicpsi - ctheta * sphispsi); x[1] = T(-sphicpsi - ctheta * cphispsi); x[2] = T(stheta * spsi);
    y[0] = T(ctheta * sphicpsi + cphispsi); y[1] = T(ctheta * cphicpsi - sphispsi); y[2] = T(-stheta * cpsi);
    z[0] = T(stheta * sphi); z[1] = T(stheta * cphi); z[2] = T(ctheta);
}

// ---------------------------------------------------------------- anisotropies
// Problems/Anisotropy/UniaxialAnisotropy.h:71-150
template <class T>
struct Uniaxial {
    T prefactorField;   // -2K/Ms   (:71-77)
    T prefactorTorque;  // -2K*V    (:79-85)
    void init(double K, double Ms, double V) {
        prefactorField = T(-2.0 * K / Ms);
        prefactorTorque = T(-2.0 * K * V);
    }
    void prepareField(const V3<T>&, const V3<T>&, const V3<T>&, const V3<T>&) const {}
    V3<T> getAnisotropyField(const V3<T>& ei, const V3<T>&, const V3<T>&, const V3<T>& ni) const {
        return (prefactorField * dot(ei, ni)) * ni;  // :140-144
    }
    V3<T> getEffTorque(const V3<T>& ei, const V3<T>&, const V3<T>&, const V3<T>& ni, const T*, const T*) const {
        return cross(ni, (prefactorTorque * dot(ei, ni)) * ei);  // :146-150
    }
    M3<T> getJacobiAnisotropyField(const V3<T>&, const V3<T>&, const V3<T>&, const V3<T>& zi) const {
        return outer(prefactorField * zi, zi);  // :130-137
    }
    // the reference's uniaxial Jacobian is already the exact derivative
    M3<T> getJacobiAnisotropyFieldExact(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {
        return getJacobiAnisotropyField(ei, xi, yi, zi);
    }
};

// Problems/Anisotropy/CubicAnisotropy.h:92-236
template <class T>
struct Cubic {
    T K1_MS;  // -2 K1 / Ms   (:93)
    T K1VM;   // -2 K1 V      (:94)
    mutable T c1m, c2m, c3m, c1m_2, c2m_2, c3m_2;
    void init(double K, double Ms, double V) {
        K1_MS = T(-2.0 * K / Ms);
        K1VM = T(-2.0 * K * V);
    }
    void prepareField(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {  // :110-121
        c1m = dot(ei, xi); c2m = dot(ei, yi); c3m = dot(ei, zi);
        c1m_2 = c1m * c1m; c2m_2 = c2m * c2m; c3m_2 = c3m * c3m;
    }
    V3<T> getAnisotropyField(const V3<T>&, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {  // :133-146
        return K1_MS * (((c2m_2 + c3m_2) * c1m) * xi + ((c1m_2 + c3m_2) * c2m) * yi + ((c1m_2 + c2m_2) * c3m) * zi);
    }
    // statesin/statecos: sines and cosines of the Brown Euler angles (:162-193)
    V3<T> getEffTorque(const V3<T>& ei, const V3<T>&, const V3<T>&, const V3<T>& zi, const T* statesin, const T* statecos) const {
        const T& ctheta = statecos[1]; const T& cpsi = statecos[2];
        const T& stheta = statesin[1]; const T& spsi = statesin[2];
        V3<T> theta; theta[0] = ctheta * spsi; theta[1] = -ctheta * cpsi; theta[2] = -stheta;
        const V3<T> symetric = ei * (c3m * (c1m_2 + c2m_2));
        const V3<T> symetricresult = cross(zi, symetric);
        const V3<T> asymetricdir = (theta * ctheta) * (T(1.0) / stheta) + zi;
        const T asymetricterm = c1m * c2m * (c2m_2 - c1m_2);
        return K1VM * (symetricresult + asymetricterm * asymetricdir);
    }
    M3<T> getJacobiAnisotropyField(const V3<T>&, const V3<T>&, const V3<T>&, const V3<T>&) const {
        return M3<T>::identity();  // placeholder Jacobian in the reference (:228-236)
    }
    // exact derivative of getAnisotropyField (:133-146): with c_i = m.a_i,
    // dH/dm = K1_MS * sum_i a_i [ (c_j^2 + c_k^2) a_i + 2 c_i c_j a_j + 2 c_i c_k a_k ]^T
    M3<T> getJacobiAnisotropyFieldExact(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {
        const V3<T> ax[3] = {xi, yi, zi};
        const T c[3] = {dot(ei, xi), dot(ei, yi), dot(ei, zi)};
        M3<T> J = M3<T>::zero();
        for (int i = 0; i < 3; ++i) {
            const int j = (i + 1) % 3, k = (i + 2) % 3;
            const V3<T> row = (c[j] * c[j] + c[k] * c[k]) * ax[i] + (T(2.0) * c[i] * c[j]) * ax[j] +
                              (T(2.0) * c[i] * c[k]) * ax[k];
            J = J + outer(ax[i], row);
        }
        return K1_MS * J;
    }
};

// ---------------------------------------------------------------- per-particle inputs
struct ParticleIn {
    double radius, Ms, alpha, gamma, K, rh, viscosity, temperature;
    double euler[3];
    double mag[3];
    double K2 = 0.0;                   // uniaxial+cubic: K_cubic
    double urot[3] = {0.0, 0.0, 0.0};  // uniaxial+cubic: Uniaxial_Rotation (Euler ZXZ)
};

template <class T> M3<T> transpose(const M3<T>& m) {
    M3<T> r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r(i, j) = m(j, i); return r;
}

// Problems/Anisotropy/UniaxialCubicAnisotropy.hpp:38-133: a uniaxial part whose axis is
// R^T z (R from Uniaxial_Rotation, calcRotation :57-83) and a cubic part on the body axes.
// The reference takes the uniaxial torque of R m on the unrotated z (:112-121) and the
// uniaxial Jacobian on the unrotated z (:125-131); both are restated as written.
template <class T>
struct UniaxialCubic {
    Uniaxial<T> uni;
    Cubic<T> cub;
    M3<T> rot;
    void init(const ParticleIn& p, double V) {
        uni.init(p.K, p.Ms, V);
        cub.init(p.K2, p.Ms, V);
        const double sphi = std::sin(p.urot[0]), cphi = std::cos(p.urot[0]);
        const double st = std::sin(p.urot[1]), ct = std::cos(p.urot[1]);
        const double sps = std::sin(p.urot[2]), cps = std::cos(p.urot[2]);
        const double cc = cphi * cps, sc = sphi * cps, cs = cphi * sps, ss = sphi * sps;
        const double r[3][3] = {{cc - ct * ss, -sc - ct * cs, st * sps},
                                {ct * sc + cs, ct * cc - ss, -st * cps},
                                {st * sphi, st * cphi, ct}};
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) rot(i, j) = T(r[i][j]);
    }
    void prepareField(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {
        cub.prepareField(ei, xi, yi, zi);  // the uniaxial part prepares nothing
    }
    V3<T> getAnisotropyField(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {
        return uni.getAnisotropyField(ei, xi, yi, transpose(rot) * zi) + cub.getAnisotropyField(ei, xi, yi, zi);
    }
    V3<T> getEffTorque(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi, const T* s, const T* c) const {
        return uni.getEffTorque(rot * ei, xi, yi, zi, s, c) + cub.getEffTorque(ei, xi, yi, zi, s, c);
    }
    M3<T> getJacobiAnisotropyField(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {
        return uni.getJacobiAnisotropyField(ei, xi, yi, zi) + cub.getJacobiAnisotropyField(ei, xi, yi, zi);
    }
    M3<T> getJacobiAnisotropyFieldExact(const V3<T>& ei, const V3<T>& xi, const V3<T>& yi, const V3<T>& zi) const {
        return uni.getJacobiAnisotropyFieldExact(ei, xi, yi, transpose(rot) * zi) + cub.getJacobiAnisotropyFieldExact(ei, xi, yi, zi);
    }
};
template <class T> void init_anisotropy(Uniaxial<T>& a, const ParticleIn& p, double V) { a.init(p.K, p.Ms, V); }
template <class T> void init_anisotropy(Cubic<T>& a, const ParticleIn& p, double V) { a.init(p.K, p.Ms, V); }
template <class T> void init_anisotropy(UniaxialCubic<T>& a, const ParticleIn& p, double V) { a.init(p, V); }
struct ProblemCfg {
    bool useRot = false;       double minAngle = 0.0;       // NeelSpherical
    bool useBrownRot = false;  double brownMinAngle = 0.0;  // BrownAndNeelEulerSpherical
    bool useNeelRot = false;   double neelMinAngle = 0.0;
    bool simpleModel = false;                               // BrownAndNeel (Cartesian)
};

}  // namespace orc
