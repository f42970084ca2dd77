// oracle_problems.hpp — restatement of the four SDE problems (test infrastructure only).
// Method names follow the reference's CRTP contract
// (SDEFramework/GeneralSDEProblem.h:116-143) so each function can be read
// side by side with the cited reference lines.
#pragma once

#include "oracle_core.hpp"

namespace orc {

using std::abs;
using std::acos;
using std::atan2;
using std::cos;
using std::fmod;
using std::isinf;
using std::sin;
using std::sqrt;

// ====================================================================== Neel (Cartesian)
// Problems/NeelRelaxation.h:24-291, dimensions <3,3,3> (:24-25)
template <class T, class Aniso>
struct NeelProblem {
    static constexpr int D = 3, M = 3, OUT = 3;
    static constexpr bool HasJacobian = true;
    using Dep = Vec<T, 3>;
    T NeelFactor1, NeelFactor2, DriftPrefactor, NoisePrefactor, Damping;
    V3<T> xAxis, yAxis, zAxis;
    Aniso mAnisotropy;
    double moment;  // Ms*V, getWeighting (:287-291)

    void init(const ParticleIn& p, const ProblemCfg&) {
        const NeelParamsD np = calc_neel_params(p.radius, p.Ms, p.alpha, p.gamma, p.temperature);
        NeelFactor1 = T(np.NeelFactor1); NeelFactor2 = T(np.NeelFactor2);
        DriftPrefactor = T(np.DriftPrefactor); NoisePrefactor = T(np.NoisePrefactor); Damping = T(np.Damping);
        euler_to_axes<T>(p.euler, xAxis, yAxis, zAxis);  // calculateParticleAxes (:223-261)
        const double V = sphere_volume(p.radius);
        init_anisotropy(mAnisotropy, p, V);
        moment = V * p.Ms;
    }
    // getStart (:263-285): the given magnetisation direction, normalised
    Dep getStart(const ParticleIn& p) const {
        const double n = std::sqrt(p.mag[0] * p.mag[0] + p.mag[1] * p.mag[1] + p.mag[2] * p.mag[2]);
        Dep r; for (int i = 0; i < 3; ++i) r[i] = T(p.mag[i] / n); return r;
    }
    void weighting(double* w) const { for (int i = 0; i < OUT; ++i) w[i] = moment; }

    void prepareCalculations(Dep&) {}
    void recomputeCache(const Dep&) {}
    void finishCalculations(Dep&) const {}
    void prepareJacobiCalculations(const Dep&) {}
    template <class J> void finishJacobiCalculations(J&) const {}

    // :92-109
    Mat<T, 3, 3> getStochasticMatrix(const Dep& yi) const {
        const T pre2 = NeelFactor2 * NoisePrefactor;
        const T pre1 = NeelFactor1 * NoisePrefactor;
        Mat<T, 3, 3> S = pre2 * M3<T>::identity() - outer(pre2 * yi, yi);
        const V3<T> yi2 = pre1 * yi;
        S(0, 1) = S(0, 1) - yi2[2]; S(0, 2) = S(0, 2) + yi2[1];
        S(1, 0) = S(1, 0) + yi2[2]; S(1, 2) = S(1, 2) - yi2[0];
        S(2, 0) = S(2, 0) - yi2[1]; S(2, 1) = S(2, 1) + yi2[0];
        return S;
    }
    // :112-116
    Dep getDrift(const Dep& yi) const { return DriftPrefactor * yi; }
    // :118-128
    Dep getDeterministicVector(const Dep& yi, const V3<T>& xi) const {
        mAnisotropy.prepareField(yi, xAxis, yAxis, zAxis);
        const V3<T> Heff = mAnisotropy.getAnisotropyField(yi, xAxis, yAxis, zAxis) + xi;
        return NeelFactor1 * cross(yi, Heff) - NeelFactor2 * cross(yi, cross(yi, Heff));
    }
    // :134-171 (including the reference's -2*alpha/dt*[m]x term, :168)
    Mat<T, 3, 3> getJacobiDeterministic(const Dep& yi, const V3<T>& xi, const T& dt) const {
        const M3<T> HeffJacobi = mAnisotropy.getJacobiAnisotropyField(yi, xAxis, yAxis, zAxis);
        const M3<T> m_plus = crossmat(yi);
        mAnisotropy.prepareField(yi, xAxis, yAxis, zAxis);
        const V3<T> Heff = mAnisotropy.getAnisotropyField(yi, xAxis, yAxis, zAxis) + xi;
        M3<T> J = m_plus * HeffJacobi;
        J(0, 1) = J(0, 1) + Heff[2]; J(0, 2) = J(0, 2) - Heff[1];
        J(1, 0) = J(1, 0) - Heff[2]; J(1, 2) = J(1, 2) + Heff[0];
        J(2, 0) = J(2, 0) + Heff[1]; J(2, 1) = J(2, 1) - Heff[0];
        return NeelFactor1 * J - ((T(2.0) * Damping) / dt) * m_plus;
    }
    // :173-190
    Mat<T, 3, 3> getJacobiStochastic(const Vec<T, 3>& dW) const {
        const T pre1 = NeelFactor1 * NoisePrefactor;
        const V3<T> dw2 = (-pre1) * dW;
        M3<T> J = M3<T>::zero();
        J(0, 1) = J(0, 1) - dw2[2]; J(0, 2) = J(0, 2) + dw2[1];
        J(1, 0) = J(1, 0) + dw2[2]; J(1, 2) = J(1, 2) - dw2[0];
        J(2, 0) = J(2, 0) - dw2[1]; J(2, 1) = J(2, 1) + dw2[0];
        return J;
    }
    // :210-214
    Vec<T, OUT> calculateOutputResult(const Dep& yi) const { return yi; }
    // NeelRelaxation.h:204-208 (Eigen normalize: unchanged at |m| = 0)
    void normalize(Dep& yi) const {
        const T n2 = yi[0] * yi[0] + yi[1] * yi[1] + yi[2] * yi[2];
        if (n2 > T(0.0)) { const T n = sqrt(n2); for (int k = 0; k < 3; ++k) yi[k] = yi[k] / n; }
    }

    // Exact Jacobians (not in the reference; its versions above keep the
    // -2 alpha/dt [m]x stand-in and drop the damping and projection derivatives).
    //   a = NF1 u - NF2 m x u, u = m x Heff(m):  J_u = [m]x J_H - [Heff]x,
    //   J_a = NF1 J_u - NF2 ([m]x J_u - [u]x)
    static constexpr bool HasExactJacobian = true;
    Mat<T, 3, 3> getJacobiDeterministicExact(const Dep& yi, const V3<T>& xi) const {
        mAnisotropy.prepareField(yi, xAxis, yAxis, zAxis);
        const V3<T> Heff = mAnisotropy.getAnisotropyField(yi, xAxis, yAxis, zAxis) + xi;
        const M3<T> JH = mAnisotropy.getJacobiAnisotropyFieldExact(yi, xAxis, yAxis, zAxis);
        const M3<T> mx = crossmat(yi);
        const M3<T> Ju = mx * JH - crossmat(Heff);
        const M3<T> Jv = mx * Ju - crossmat(cross(yi, Heff));
        return NeelFactor1 * Ju - NeelFactor2 * Jv;
    }
    //   b(m) dW = pre2 (dW - m (m.dW)) + pre1 m x dW:  J = -pre2 ((m.dW) I + m dW^T) - pre1 [dW]x
    Mat<T, 3, 3> getJacobiStochasticExact(const Dep& yi, const Vec<T, 3>& dW) const {
        const T pre2 = NeelFactor2 * NoisePrefactor;
        const T pre1 = NeelFactor1 * NoisePrefactor;
        return (T(-1.0) * pre2) * (dot(yi, dW) * M3<T>::identity() + outer(yi, dW)) - pre1 * crossmat(dW);
    }
};

// ====================================================================== Neel (spherical)
// Problems/NeelRelaxationSpherical.h:29-601, dimensions <2,3,3> (:29-30)
template <class T, class Aniso>
struct NeelSphericalProblem {
    static constexpr int D = 2, M = 3, OUT = 3;
    static constexpr bool HasJacobian = true;
    static constexpr bool HasExactJacobian = false;
    using Dep = Vec<T, 2>;
    T NeelFactor1, NeelFactor2, DriftPrefactor, NoisePrefactor, Damping;
    V3<T> xAxis, yAxis, zAxis;
    Aniso mAnisotropy;
    double moment;
    bool RotateCoordinateSystem = false;
    T MinAngleBeforeRotation, MaxAngleBeforeRotation;
    // caches (:85-99)
    bool isRotated = false;
    T one_div_sin_t;
    V3<T> MagnetisationDir, e_theta, e_phi;
    Mat<T, 2, 3> ProjectionMatrix;
    Mat<T, 2, 3> Jacobi_er, Jacobi_theta, Jacobi_phi;

    void init(const ParticleIn& p, const ProblemCfg& cfg) {
        const NeelParamsD np = calc_neel_params(p.radius, p.Ms, p.alpha, p.gamma, p.temperature);
        NeelFactor1 = T(np.NeelFactor1); NeelFactor2 = T(np.NeelFactor2);
        DriftPrefactor = T(np.DriftPrefactor); NoisePrefactor = T(np.NoisePrefactor); Damping = T(np.Damping);
        euler_to_axes<T>(p.euler, xAxis, yAxis, zAxis);  // (:614-620)
        const double V = sphere_volume(p.radius);
        init_anisotropy(mAnisotropy, p, V);
        moment = V * p.Ms;
        RotateCoordinateSystem = cfg.useRot;  // (:113)
        MinAngleBeforeRotation = T(cfg.minAngle);
        MaxAngleBeforeRotation = T(kPi - cfg.minAngle);
    }
    // getStart (:518-526) with ConvertMagnetisationDirectionToSphericalCoordinates
    // (Problems/Helpers/ParticleStateInitializer.h:132-144)
    Dep getStart(const ParticleIn& p) const {
        Dep r; r[0] = T(std::acos(p.mag[2])); r[1] = T(std::atan2(p.mag[1], p.mag[0])); return r;
    }
    void weighting(double* w) const { for (int i = 0; i < OUT; ++i) w[i] = moment; }

    // :546-559
    bool needsCoordRotation(const Dep& yi) const {
        if (RotateCoordinateSystem) {
            const T& theta = yi[0];
            if (theta < MinAngleBeforeRotation || theta > MaxAngleBeforeRotation) return true;
        }
        return false;
    }
    // :568-580
    Dep Rotate2DSphericalCoordinate90DegreeAroundYAxis(const Dep& yi) const {
        const T sin_t = sin(yi[0]);
        Dep r; r[0] = acos(-cos(yi[1]) * sin_t); r[1] = atan2(sin(yi[1]) * sin_t, cos(yi[0])); return r;
    }
    // :589-602
    Dep inverseRotate2DSphericalCoordinate90DegreeAroundYAxis(const Dep& yi) const {
        const T sin_t = sin(yi[0]);
        Dep r; r[0] = acos(cos(yi[1]) * sin_t); r[1] = atan2(sin(yi[1]) * sin_t, -cos(yi[0])); return r;
    }
    // :124-237
    void prepareCalculations(Dep& yi) {
        if (needsCoordRotation(yi)) { yi = Rotate2DSphericalCoordinate90DegreeAroundYAxis(yi); isRotated = true; }
        else isRotated = false;
        recomputeCache(yi);
    }
    // the cache part of prepareCalculations (:146-236) for the current rotation state
    void recomputeCache(const Dep& yi) {
        const T sin_t = sin(yi[0]), cos_t = cos(yi[0]), sin_p = sin(yi[1]), cos_p = cos(yi[1]);
        one_div_sin_t = T(1.0) / sin_t;
        if (isinf(one_div_sin_t)) one_div_sin_t = T(0.0);
        const T& a = NeelFactor1; const T& b = NeelFactor2;
        if (!isRotated) {
            MagnetisationDir[0] = sin_t * cos_p; MagnetisationDir[1] = sin_t * sin_p; MagnetisationDir[2] = cos_t;
            e_theta[0] = cos_t * cos_p; e_theta[1] = cos_t * sin_p; e_theta[2] = -sin_t;
            e_phi[0] = -sin_p; e_phi[1] = cos_p; e_phi[2] = T(0.0);
        } else {
            MagnetisationDir[0] = -cos_t; MagnetisationDir[1] = sin_t * sin_p; MagnetisationDir[2] = sin_t * cos_p;
            e_theta[0] = sin_t; e_theta[1] = cos_t * sin_p; e_theta[2] = cos_t * cos_p;
            e_phi[0] = T(0.0); e_phi[1] = cos_p; e_phi[2] = -sin_p;
        }
        const V3<T> r0 = (-a) * e_phi + b * e_theta;
        const V3<T> r1 = one_div_sin_t * (a * e_theta + b * e_phi);
        for (int j = 0; j < 3; ++j) { ProjectionMatrix(0, j) = r0[j]; ProjectionMatrix(1, j) = r1[j]; }
        if (one_div_sin_t == T(0.0)) {
            if (!isRotated) ProjectionMatrix(1, 2) = a;  // :193-195
            else ProjectionMatrix(1, 0) = -a;            // :233-235
        }
    }
    // :239-265
    Dep getDeterministicVector(const Dep&, const V3<T>& xi) const {
        mAnisotropy.prepareField(MagnetisationDir, xAxis, yAxis, zAxis);
        const V3<T> Heff = mAnisotropy.getAnisotropyField(MagnetisationDir, xAxis, yAxis, zAxis) + xi;
        return ProjectionMatrix * Heff;
    }
    // :267-293
    Mat<T, 2, 3> getStochasticMatrix(const Dep&) const { return NoisePrefactor * ProjectionMatrix; }
    // :295-309
    Dep getDrift(const Dep&) const {
        const T cos_t = isRotated ? -MagnetisationDir[0] : MagnetisationDir[2];
        Dep d; d[0] = T(-0.5) * DriftPrefactor * cos_t * one_div_sin_t; d[1] = T(0.0); return d;
    }
    // :312-337
    void prepareJacobiCalculations(const Dep&) {
        const T cos_t = isRotated ? -MagnetisationDir[0] : MagnetisationDir[2];
        const T sin_t = isRotated ? e_theta[0] : -e_theta[2];
        for (int j = 0; j < 3; ++j) {
            Jacobi_er(0, j) = e_theta[j]; Jacobi_er(1, j) = sin_t * e_phi[j];
            Jacobi_theta(0, j) = -MagnetisationDir[j]; Jacobi_theta(1, j) = cos_t * e_phi[j];
            Jacobi_phi(0, j) = T(0.0);
        }
        if (isRotated) { Jacobi_phi(1, 0) = T(0.0); Jacobi_phi(1, 1) = e_phi[2]; Jacobi_phi(1, 2) = -e_phi[1]; }
        else { Jacobi_phi(1, 0) = -e_phi[1]; Jacobi_phi(1, 1) = e_phi[0]; Jacobi_phi(1, 2) = T(0.0); }
    }
    // :340-409
    Mat<T, 2, 2> getJacobiDeterministic(const Dep&, const V3<T>& xi, const T&) const {
        const M3<T> HeffJacobi = mAnisotropy.getJacobiAnisotropyField(MagnetisationDir, xAxis, yAxis, zAxis);
        mAnisotropy.prepareField(MagnetisationDir, xAxis, yAxis, zAxis);
        const V3<T> EffField = mAnisotropy.getAnisotropyField(MagnetisationDir, xAxis, yAxis, zAxis) + xi;
        Mat<T, 2, 2> res = Mat<T, 2, 2>::zero();
        const T& a = NeelFactor1; const T& b = NeelFactor2;
        // row 0: (-a*J_phi + b*J_theta) * Heff + P_row0 * (HJ * J_er^T)
        const Mat<T, 2, 3> A0 = (-a) * Jacobi_phi + b * Jacobi_theta;
        const Vec<T, 2> part1 = A0 * EffField;
        for (int c = 0; c < 2; ++c) {
            T s = T(0.0);
            for (int k = 0; k < 3; ++k) {
                T hj = T(0.0);
                for (int l = 0; l < 3; ++l) hj = hj + HeffJacobi(k, l) * Jacobi_er(c, l);
                s = s + ProjectionMatrix(0, k) * hj;
            }
            res(0, c) = part1[c] + s;
        }
        if (!isinf(one_div_sin_t)) {
            const T cos_t = isRotated ? -MagnetisationDir[0] : MagnetisationDir[2];
            const T jac_sin_t0 = one_div_sin_t * one_div_sin_t * cos_t;  // Jac_Sin_t = (.., 0)
            const Mat<T, 2, 3> B1 = one_div_sin_t * (a * Jacobi_theta + b * Jacobi_phi);
            const V3<T> ab = a * e_theta + b * e_phi;
            for (int c = 0; c < 2; ++c) {
                T s = T(0.0);
                for (int k = 0; k < 3; ++k) s = s + EffField[k] * (B1(c, k) - (c == 0 ? ab[k] * jac_sin_t0 : T(0.0)));
                T s2 = T(0.0);
                for (int k = 0; k < 3; ++k) {
                    T ph = T(0.0);
                    for (int l = 0; l < 3; ++l) ph = ph + ProjectionMatrix(1, l) * HeffJacobi(l, k);
                    s2 = s2 + ph * Jacobi_er(c, k);
                }
                res(1, c) = s + s2;
            }
        }
        return res;
    }
    // :411-432
    Mat<T, 2, 2> getJacobiStochastic(const Vec<T, 3>& dW) const {
        Mat<T, 2, 2> res = Mat<T, 2, 2>::zero();
        const T& a = NeelFactor1; const T& b = NeelFactor2;
        const T cos_t = isRotated ? -MagnetisationDir[0] : MagnetisationDir[2];
        const Mat<T, 2, 3> A0 = NoisePrefactor * ((-a) * Jacobi_phi + b * Jacobi_theta);
        const Vec<T, 2> r0 = A0 * dW;
        res(0, 0) = r0[0]; res(0, 1) = r0[1];
        if (!isinf(one_div_sin_t)) {
            const T jac_sin_t0 = one_div_sin_t * one_div_sin_t * cos_t;
            const Mat<T, 2, 3> B1 = one_div_sin_t * (a * Jacobi_theta + b * Jacobi_phi);
            const V3<T> ab = a * e_theta + b * e_phi;
            for (int c = 0; c < 2; ++c) {
                T s = T(0.0);
                for (int k = 0; k < 3; ++k) s = s + dW[k] * NoisePrefactor * (B1(c, k) - (c == 0 ? ab[k] * jac_sin_t0 : T(0.0)));
                res(1, c) = s;
            }
        }
        return res;
    }
    // :441-471
    void finishCalculations(Dep& yi) const {
        if (isRotated) yi = inverseRotate2DSphericalCoordinate90DegreeAroundYAxis(yi);
        else { yi[0] = fmod(yi[0], T(kTwoPi)); yi[1] = fmod(yi[1], T(kTwoPi)); }
    }
    // :473-497
    void finishJacobiCalculations(Mat<T, 2, 2>& jacobi) const {
        if (isRotated) {
            const T m_cos_t = MagnetisationDir[0];
            const T sin_t = e_theta[0];
            const T cos_p = e_phi[1];
            const T m_sin_p = e_phi[2];
            Mat<T, 2, 2> J;
            const T factor = T(1.0) / sqrt(T(1.0) - sin_t * sin_t * cos_p * cos_p);
            J(0, 0) = factor * m_cos_t * cos_p;
            J(0, 1) = m_sin_p;
            J(1, 0) = -factor * one_div_sin_t * m_sin_p;
            J(1, 1) = one_div_sin_t * m_cos_t * cos_p;
            jacobi = jacobi * J;
        }
    }
    // :500-516
    Vec<T, OUT> calculateOutputResult(const Dep& yi) const {
        const T sin_t = sin(yi[0]), cos_t = cos(yi[0]), sin_p = sin(yi[1]), cos_p = cos(yi[1]);
        Vec<T, 3> o; o[0] = sin_t * cos_p; o[1] = sin_t * sin_p; o[2] = cos_t; return o;
    }
    void normalize(Dep&) const {}  // spherical coordinates: no-op in the reference
};

// ====================================================================== Brown + Neel, Euler/spherical
// Problems/BrownAndNeelRelaxationEulerSpherical.h:36-899, dimensions <5,3,6> (:36-37)
template <class T, class Aniso>
struct BrownNeelEulerProblem {
    static constexpr int D = 5, M = 6, OUT = 9;
    static constexpr bool HasJacobian = false;  // assert(false) in the reference (:605-626)
    static constexpr bool HasExactJacobian = false;
    using Dep = Vec<T, 5>;
    T a_, b_, DN, c_, DB, cF, MagneticMoment;  // NeelFactor1/2, NoisePrefactor, BrownPrefactor/Diffusion, Brown_F_Noise
    Aniso mAnisotropy;
    double moment;
    bool brownRot = false, neelRot = false;
    T brownMin, brownMax, neelMin, neelMax;
    // caches (:96-114)
    T S[5], C[5];
    V3<T> MagnetisationDir;
    bool bIsRotated = false, nIsRotated = false;
    T csctheta, one_div_sin_t;
    M3<T> EulerRotationMatrix, EulerProjectionMatrix;
    Mat<T, 2, 3> SphericalProjectionMatrix;

    void init(const ParticleIn& p, const ProblemCfg& cfg) {
        const NeelParamsD np = calc_neel_params(p.radius, p.Ms, p.alpha, p.gamma, p.temperature);
        const BrownParamsD bp = calc_brown_params(p.rh, p.viscosity, p.temperature);
        a_ = T(np.NeelFactor1); b_ = T(np.NeelFactor2); DN = T(np.NoisePrefactor);
        c_ = T(bp.BrownPrefactor); DB = T(bp.BrownDiffusion); cF = T(bp.Brown_F_Noise);
        const double V = sphere_volume(p.radius);
        moment = V * p.Ms;
        MagneticMoment = T(moment);
        init_anisotropy(mAnisotropy, p, V);
        brownRot = cfg.useBrownRot; brownMin = T(cfg.brownMinAngle); brownMax = T(kPi - cfg.brownMinAngle);  // :129
        neelRot = cfg.useNeelRot; neelMin = T(cfg.neelMinAngle); neelMax = T(kPi - cfg.neelMinAngle);        // :130
    }
    // getStart (:741-753): Euler angles as given, magnetisation converted to spherical
    Dep getStart(const ParticleIn& p) const {
        Dep r;
        for (int i = 0; i < 3; ++i) r[i] = T(p.euler[i]);
        r[3] = T(std::acos(p.mag[2])); r[4] = T(std::atan2(p.mag[1], p.mag[0]));
        return r;
    }
    void weighting(double* w) const { for (int i = 0; i < OUT; ++i) w[i] = moment; }  // :755-759

    // :770-786
    bool needsNeelCoordRotation(const Dep& yi) const {
        if (neelRot) { const T t = abs(yi[3]); if (t < neelMin) return true; else if (t > neelMax) return true; }
        return false;
    }
    // :796-813
    bool needsBrownCoordRotation(const Dep& yi) const {
        if (brownRot) { const T t = abs(yi[1]); if (t < brownMin) return true; else if (t > brownMax) return true; }
        return false;
    }
    // :823-834
    void rotNeel(T& th, T& ph) const {
        const T sin_t = sin(th); const T nt = acos(-cos(ph) * sin_t); const T np = atan2(sin(ph) * sin_t, cos(th)); th = nt; ph = np;
    }
    // :844-856
    void invRotNeel(T& th, T& ph) const {
        const T sin_t = sin(th); const T nt = acos(cos(ph) * sin_t); const T np = atan2(sin(ph) * sin_t, -cos(th)); th = nt; ph = np;
    }
    // :859-878
    void EulertoEulerRotated(T* e) const {
        const T S0 = sin(e[0]), S1 = sin(e[1]), S2 = sin(e[2]), C0 = cos(e[0]), C1 = cos(e[1]), C2 = cos(e[2]);
        const T newphi = atan2(-C2 * C0 + C1 * S0 * S2, S0 * C2 + C1 * C0 * S2);
        const T newtheta = acos(-S1 * S2);
        const T newpsi = atan2(C1, C2 * S1);
        e[0] = newphi; e[1] = newtheta; e[2] = newpsi;
    }
    // :880-899
    void EulerRotatedtoEuler(T* e) const {
        const T S0 = sin(e[0]), S1 = sin(e[1]), S2 = sin(e[2]), C0 = cos(e[0]), C1 = cos(e[1]), C2 = cos(e[2]);
        const T newphi = atan2(C0 * C2 - C1 * S0 * S2, -C2 * S0 - C1 * C0 * S2);
        const T newtheta = acos(S1 * S2);
        const T newpsi = atan2(-C1, C2 * S1);
        e[0] = newphi; e[1] = newtheta; e[2] = newpsi;
    }
    // :141-361
    void prepareCalculations(Dep& yi) {
        if (needsBrownCoordRotation(yi)) { EulertoEulerRotated(&yi[0]); bIsRotated = true; } else bIsRotated = false;
        if (needsNeelCoordRotation(yi)) { rotNeel(yi[3], yi[4]); nIsRotated = true; } else nIsRotated = false;
        recomputeCache(yi);
    }
    void recomputeCache(const Dep& yi) {
        for (int i = 0; i < 5; ++i) { S[i] = sin(yi[i]); C[i] = cos(yi[i]); }
        const T& cphi = C[0]; const T& ctheta = C[1]; const T& cpsi = C[2];
        const T& sphi = S[0]; const T& stheta = S[1]; const T& spsi = S[2];
        const T cphicpsi = cphi * cpsi, sphicpsi = sphi * cpsi, cphispsi = cphi * spsi, sphispsi = sphi * spsi;
        const T cthetacpsi = ctheta * cpsi, cthetaspsi = ctheta * spsi;
        M3<T>& R = EulerRotationMatrix; M3<T>& E = EulerProjectionMatrix;
        csctheta = T(1.0) / stheta;
        if (isinf(csctheta)) csctheta = T(0.0);
        if (!bIsRotated) {  // :183-238
            R(0, 0) = cphicpsi - ctheta * sphispsi; R(0, 1) = -sphicpsi - ctheta * cphispsi; R(0, 2) = stheta * spsi;
            R(1, 0) = ctheta * sphicpsi + cphispsi; R(1, 1) = ctheta * cphicpsi - sphispsi; R(1, 2) = -stheta * cpsi;
            R(2, 0) = stheta * sphi; R(2, 1) = stheta * cphi; R(2, 2) = ctheta;
            E(0, 0) = spsi * csctheta; E(1, 0) = cpsi; E(2, 0) = -cthetaspsi * csctheta;
            E(0, 1) = -cpsi * csctheta; E(1, 1) = spsi; E(2, 1) = cthetacpsi * csctheta;
            E(0, 2) = T(0.0); E(1, 2) = T(0.0); E(2, 2) = T(1.0);
        } else {  // :239-304
            R(0, 0) = -stheta * sphi; R(0, 1) = -stheta * cphi; R(0, 2) = -ctheta;
            R(1, 0) = ctheta * sphicpsi + cphispsi; R(1, 1) = ctheta * cphicpsi - sphispsi; R(1, 2) = -stheta * cpsi;
            R(2, 0) = cphicpsi - ctheta * sphispsi; R(2, 1) = -sphicpsi - ctheta * cphispsi; R(2, 2) = stheta * spsi;
            E(0, 0) = T(0.0); E(1, 0) = T(0.0); E(2, 0) = T(-1.0);
            E(0, 1) = -cpsi * csctheta; E(1, 1) = spsi; E(2, 1) = cthetacpsi * csctheta;
            E(0, 2) = spsi * csctheta; E(1, 2) = cpsi; E(2, 2) = -cthetaspsi * csctheta;
        }
        const T& cos_t = C[3]; const T& cos_p = C[4]; const T& sin_t = S[3]; const T& sin_p = S[4];
        Mat<T, 2, 3>& P = SphericalProjectionMatrix;
        one_div_sin_t = T(1.0) / sin_t;
        if (isinf(one_div_sin_t)) one_div_sin_t = T(0.0);
        if (!nIsRotated) {  // :307-330
            MagnetisationDir[0] = sin_t * cos_p; MagnetisationDir[1] = sin_t * sin_p; MagnetisationDir[2] = cos_t;
            P(0, 0) = -sin_p; P(1, 0) = -cos_p * cos_t * one_div_sin_t;
            P(0, 1) = cos_p;  P(1, 1) = -sin_p * cos_t * one_div_sin_t;
            P(0, 2) = T(0.0); P(1, 2) = T(1.0);
        } else {  // :331-360
            MagnetisationDir[0] = -cos_t; MagnetisationDir[1] = sin_t * sin_p; MagnetisationDir[2] = sin_t * cos_p;
            P(0, 0) = T(0.0); P(1, 0) = T(-1.0);
            P(0, 1) = cos_p;  P(1, 1) = -sin_p * cos_t * one_div_sin_t;
            P(0, 2) = -sin_p; P(1, 2) = -cos_p * cos_t * one_div_sin_t;
        }
    }
    V3<T> col(const M3<T>& m, int c) const { V3<T> v; v[0] = m(0, c); v[1] = m(1, c); v[2] = m(2, c); return v; }
    // :363-425
    Dep getDeterministicVector(const Dep&, const V3<T>& xi) const {
        const V3<T> xAxis = col(EulerRotationMatrix, 0), yAxis = col(EulerRotationMatrix, 1), zAxis = col(EulerRotationMatrix, 2);
        mAnisotropy.prepareField(MagnetisationDir, xAxis, yAxis, zAxis);
        const V3<T> Heff = mAnisotropy.getAnisotropyField(MagnetisationDir, xAxis, yAxis, zAxis) + xi;
        const V3<T> Teff = mAnisotropy.getEffTorque(MagnetisationDir, xAxis, yAxis, zAxis, S, C);
        const T& c = c_;
        const T d = c * MagneticMoment;
        const V3<T> mxHeff = cross(MagnetisationDir, Heff);
        const V3<T> omegabrown = c * Teff + d * mxHeff;
        const V3<T> brownres = EulerProjectionMatrix * omegabrown;
        const V3<T> omeganeel = (-a_) * Heff + (b_ + d) * mxHeff + c * Teff;
        const Vec<T, 2> neelres = SphericalProjectionMatrix * omeganeel;
        Dep r; r[0] = brownres[0]; r[1] = brownres[1]; r[2] = brownres[2]; r[3] = neelres[0]; r[4] = neelres[1];
        return r;
    }
    // :427-497
    Mat<T, 5, 6> getStochasticMatrix(const Dep&) const {
        Mat<T, 5, 6> R = Mat<T, 5, 6>::zero();
        const M3<T> BrownTorqueNoise = cF * EulerProjectionMatrix;
        const T& c = c_;
        const T d = c * MagneticMoment;
        const V3<T> tmp = (d * DN) * MagnetisationDir;
        const M3<T> BrownFieldNoise = EulerProjectionMatrix * crossmat(tmp);
        const Mat<T, 2, 3> NeelTorqueNoise = SphericalProjectionMatrix * (cF * M3<T>::identity());
        const V3<T> tmp2 = ((b_ + d) * DN) * MagnetisationDir;
        const M3<T> Mt = crossmat(tmp2) - (a_ * DN) * M3<T>::identity();
        const Mat<T, 2, 3> NeelFieldNoise = SphericalProjectionMatrix * Mt;
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { R(i, j) = BrownTorqueNoise(i, j); R(i, j + 3) = BrownFieldNoise(i, j); }
        for (int i = 0; i < 2; ++i) for (int j = 0; j < 3; ++j) { R(3 + i, j) = NeelTorqueNoise(i, j); R(3 + i, j + 3) = NeelFieldNoise(i, j); }
        return R;
    }
    // :499-601
    Dep getDrift(const Dep& yi) const {
        const T& a = a_; const T& b = b_; const T& c = c_;
        const T d = c * MagneticMoment;
        const T& ctheta = C[1]; const T& cpsi = C[2]; const T& spsi = S[2];
        const T& cos_t = C[3]; const T& cos_p = C[4]; const T& sin_t = S[3]; const T& sin_p = S[4];
        const T DN_2 = DN * DN, DB_2 = DB * DB;
        const T c_2_half = T(0.5) * c * c;
        const T d_2_fourth = T(0.25) * d * d;
        const T a_d = a * d;
        const T bpd = b + d;
        Dep r;
        if ((!bIsRotated && !nIsRotated) || (bIsRotated && nIsRotated)) {  // :542-558
            const T cotb = csctheta * ctheta;
            const T cos_2t = cos_t * cos_t - sin_t * sin_t;
            const T sin_2t = T(2.0) * cos_t * sin_t;
            const T sin_t_2 = sin_t * sin_t;
            const T cos_phinmpsib = cos_p * cpsi + spsi * sin_p;
            const T sin_phinmpsib = cpsi * sin_p - cos_p * spsi;
            const T twophineelminuspsibrown = T(2.0) * (yi[4] - yi[2]);
            const T cos_2phinmpsib = cos(twophineelminuspsibrown);
            const T sin_2phinmpsib = sin(twophineelminuspsibrown);
            r[0] = -DN_2 * csctheta * sin_t * (-a * d * sin_phinmpsib + T(2.0) * d_2_fourth * (cos_t * cos_phinmpsib + cotb * sin_t * sin_2phinmpsib));
            r[1] = c_2_half * DB_2 * cotb - DN_2 * a_d * (cos_phinmpsib * sin_t) + d_2_fourth * DN_2 * (T(0.5) * (T(3.0) + cos_2t + T(2.0) * cos_2phinmpsib * sin_t_2) * cotb - sin_2t * sin_phinmpsib);
            r[2] = -DN_2 * (a_d * (cos_t + sin_t * cotb * sin_phinmpsib) - d_2_fourth * sin_t * (T(2.0) * cos_t * cotb * cos_phinmpsib + (T(-1.0) + T(2.0) * csctheta * csctheta) * sin_t * sin_2phinmpsib));
        } else if (bIsRotated) {  // :559-576
            const T sin_2t = T(2.0) * cos_t * sin_t;
            const T sin_t_2 = sin_t * sin_t;
            const T cpsi_2 = cpsi * cpsi, spsi_2 = spsi * spsi;
            const T c2psi = cpsi_2 - spsi_2, s2psi = T(2.0) * cpsi * spsi;
            const T sin_2p = T(2.0) * cos_p * sin_p;
            const T cotb = csctheta * ctheta;
            const T cos_t_2 = cos_t * cos_t, sin_p_2 = sin_p * sin_p, cos_p_2 = cos_p * cos_p;
            r[0] = DN_2 * csctheta * (a_d * (-spsi * cos_t + sin_p * cpsi * sin_t) + T(2.0) * d_2_fourth * (-c2psi * cotb * sin_2t * sin_p + cos_p * sin_t * (cos_t * cpsi + sin_t * sin_p * spsi) + cotb * s2psi * (cos_t_2 - sin_t_2 * sin_p_2)));
            r[1] = c_2_half * DB_2 * cotb + DN_2 * (a_d * (-cos_t * cpsi - spsi * sin_t * sin_p) + d_2_fourth * (T(2.0) * cpsi_2 * cotb * (cos_t_2 + cos_p_2 * sin_t_2) + cpsi * sin_t_2 * sin_2p + T(2.0) * spsi * (-sin_t * cos_t * cos_p + cotb * sin_t_2 * spsi) + cotb * sin_2t * sin_p * s2psi));
            r[2] = DN_2 * (a_d * (sin_t * cos_p - cpsi * cotb * sin_t * sin_p + cotb * cos_t * spsi) - d_2_fourth * (cos_t * cpsi + sin_t * sin_p * spsi) * (T(2.0) * cos_p * cotb * sin_t - (T(3.0) + c2psi) * csctheta * csctheta * (cpsi * sin_t * sin_p - cos_t * spsi)));
        } else {  // only Neel rotated, :577-594
            const T sin_2t = T(2.0) * cos_t * sin_t;
            const T sin_t_2 = sin_t * sin_t;
            const T cpsi_2 = cpsi * cpsi, spsi_2 = spsi * spsi;
            const T c2psi = cpsi_2 - spsi_2, s2psi = T(2.0) * cpsi * spsi;
            const T sin_2p = T(2.0) * cos_p * sin_p;
            const T cotb = csctheta * ctheta;
            const T cos_t_2 = cos_t * cos_t, sin_p_2 = sin_p * sin_p, cos_p_2 = cos_p * cos_p;
            r[0] = DN_2 * csctheta * (a_d * (spsi * cos_t + sin_p * cpsi * sin_t) + T(2.0) * d_2_fourth * (c2psi * cotb * sin_2t * sin_p + cos_p * sin_t * (cos_t * cpsi - sin_t * sin_p * spsi) + cotb * s2psi * (cos_t_2 - sin_t_2 * sin_p_2)));
            r[1] = c_2_half * DB_2 * cotb + DN_2 * (a_d * (+cos_t * cpsi - spsi * sin_t * sin_p) + d_2_fourth * (T(2.0) * cpsi_2 * cotb * (cos_t_2 + cos_p_2 * sin_t_2) - cpsi * sin_t_2 * sin_2p + T(2.0) * spsi * (-sin_t * cos_t * cos_p + cotb * sin_t_2 * spsi) - cotb * sin_2t * sin_p * s2psi));
            r[2] = DN_2 * (a_d * (-sin_t * cos_p - cpsi * cotb * sin_t * sin_p - cotb * cos_t * spsi) - d_2_fourth * (cos_t * cpsi - sin_t * sin_p * spsi) * (T(2.0) * cos_p * cotb * sin_t + (T(3.0) + c2psi) * csctheta * csctheta * (cpsi * sin_t * sin_p + cos_t * spsi)));
        }
        r[3] = (c_2_half * DB_2 + T(0.5) * (a * a + bpd * bpd) * DN_2) * one_div_sin_t * cos_t;  // :597
        r[4] = T(0.0);
        return r;
    }
    void prepareJacobiCalculations(const Dep&) {}
    template <class J> void finishJacobiCalculations(J&) const {}
    // :634-665
    void finishCalculations(Dep& yi) const {
        if (bIsRotated) EulerRotatedtoEuler(&yi[0]);
        else { yi[0] = fmod(yi[0], T(kTwoPi)); yi[1] = fmod(yi[1], T(kTwoPi)); yi[2] = fmod(yi[2], T(kTwoPi)); }
        if (nIsRotated) invRotNeel(yi[3], yi[4]);
        else { yi[3] = fmod(yi[3], T(kTwoPi)); yi[4] = fmod(yi[4], T(kTwoPi)); }
    }
    // :673-735
    Vec<T, OUT> calculateOutputResult(const Dep& yi) const {
        T s[5], c[5];
        for (int i = 0; i < 5; ++i) { s[i] = sin(yi[i]); c[i] = cos(yi[i]); }
        const T& cphi = c[0]; const T& ctheta = c[1]; const T& cpsi = c[2];
        const T& sphi = s[0]; const T& stheta = s[1]; const T& spsi = s[2];
        const T cphicpsi = cphi * cpsi, sphicpsi = sphi * cpsi, cphispsi = cphi * spsi, sphispsi = sphi * spsi;
        Vec<T, OUT> o;
        o[0] = cphicpsi - ctheta * sphispsi; o[1] = ctheta * sphicpsi + cphispsi; o[2] = stheta * sphi;
        o[3] = -sphicpsi - ctheta * cphispsi; o[4] = ctheta * cphicpsi - sphispsi; o[5] = stheta * cphi;
        o[6] = s[3] * c[4]; o[7] = s[3] * s[4]; o[8] = c[3];
        return o;
    }
    void normalize(Dep&) const {}  // spherical coordinates: no-op in the reference
};

// ====================================================================== Brown + Neel (Cartesian)
// Problems/BrownAndNeelRelaxation.h:68-187, Problems/BrownAndNeelRelaxation.inl:40-324
template <class T, class Aniso, bool IsCubic>
struct BrownNeelProblem {
    static constexpr int D = 6, M = 6, OUT = 6;
    static constexpr bool HasJacobian = true;
    static constexpr bool HasExactJacobian = false;
    using Dep = Vec<T, 6>;
    T a_, b_, DN, c_, cF, MagneticMoment;
    Aniso mAnisotropy;
    double moment;
    bool simple = false;

    void init(const ParticleIn& p, const ProblemCfg& cfg) {
        const NeelParamsD np = calc_neel_params(p.radius, p.Ms, p.alpha, p.gamma, p.temperature);
        const BrownParamsD bp = calc_brown_params(p.rh, p.viscosity, p.temperature);
        a_ = T(np.NeelFactor1); b_ = T(np.NeelFactor2); DN = T(np.NoisePrefactor);
        c_ = T(bp.BrownPrefactor); cF = T(bp.Brown_F_Noise);
        const double V = sphere_volume(p.radius);
        moment = V * p.Ms;
        MagneticMoment = T(moment);
        init_anisotropy(mAnisotropy, p, V);
        simple = cfg.simpleModel;
    }
    // getStart (.inl:278-324) with Use_random_* = false
    Dep getStart(const ParticleIn& p) const {
        const double a = p.euler[0], b = p.euler[1], g = p.euler[2];
        double n[3] = {std::cos(a) * std::cos(g) - std::sin(a) * std::cos(b) * std::sin(g),
                       -std::cos(a) * std::sin(g) - std::sin(a) * std::cos(b) * std::cos(g),
                       std::sin(a) * std::sin(b)};
        double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        double mm = std::sqrt(p.mag[0] * p.mag[0] + p.mag[1] * p.mag[1] + p.mag[2] * p.mag[2]);
        Dep r;
        for (int i = 0; i < 3; ++i) { r[i] = T(n[i] / nn); r[3 + i] = T(p.mag[i] / mm); }
        return r;
    }
    // .h:152-159: 1 for the axis, Ms*V for the magnetisation
    void weighting(double* w) const { for (int i = 0; i < 3; ++i) { w[i] = 1.0; w[3 + i] = moment; } }

    void prepareCalculations(Dep&) {}
    void recomputeCache(const Dep&) {}
    void finishCalculations(Dep&) const {}
    void prepareJacobiCalculations(const Dep&) {}
    template <class J> void finishJacobiCalculations(J&) const {}

    static V3<T> head(const Dep& y) { V3<T> v; v[0] = y[0]; v[1] = y[1]; v[2] = y[2]; return v; }
    static V3<T> tail(const Dep& y) { V3<T> v; v[0] = y[3]; v[1] = y[4]; v[2] = y[5]; return v; }

    // .inl:222-271
    Dep getDeterministicVector(const Dep& yi, const V3<T>& xi) const {
        if (IsCubic) return Dep::zero();  // .inl:225-229 (not implemented in the reference)
        const V3<T> ni = head(yi), ei = tail(yi);
        const V3<T> zeroAxis = V3<T>::zero();
        mAnisotropy.prepareField(ei, zeroAxis, zeroAxis, ni);
        const V3<T> Heff = mAnisotropy.getAnisotropyField(ei, zeroAxis, zeroAxis, ni) + xi;
        T zs[3] = {T(0.0), T(0.0), T(0.0)};
        const V3<T> Teff = mAnisotropy.getEffTorque(ei, zeroAxis, zeroAxis, ni, zs, zs);
        const T& c = c_;
        const T d = c * MagneticMoment;
        const V3<T> mxHeff = cross(ei, Heff);
        const V3<T> omegabrown = c * Teff + d * mxHeff;
        const V3<T> brown = cross(omegabrown, ni);
        const V3<T> omeganeel = (-a_) * Heff + (b_ + d) * mxHeff + c * Teff;
        const V3<T> neel = cross(omeganeel, ei);
        Dep r; for (int i = 0; i < 3; ++i) { r[i] = brown[i]; r[3 + i] = neel[i]; } return r;
    }
    // .inl:40-111 (full) and :115-170 (simplified)
    Mat<T, 6, 6> getStochasticMatrix(const Dep& yi) const {
        const V3<T> ni = head(yi), ei = tail(yi);
        const T& c = c_;
        const T d = c * MagneticMoment;
        Mat<T, 6, 6> S = Mat<T, 6, 6>::zero();
        M3<T> Brown_H = M3<T>::zero(), Neel_F = M3<T>::zero();
        if (!simple) {
            const T d_H_Noise = d * DN;
            const V3<T> dni = d_H_Noise * ni;
            Brown_H = dot(dni, ei) * M3<T>::identity() - outer(ei, dni);
            Neel_F = T(-1.0) * crossmat(cF * ei);
        }
        const M3<T> Brown_F = T(-1.0) * crossmat(cF * ni);
        const M3<T> outerei = M3<T>::identity() - outer(ei, ei);
        const T pre = simple ? b_ * DN : (b_ + d) * DN;
        const M3<T> Neel_H = pre * outerei + crossmat((a_ * DN) * ei);
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
            S(i, j) = Brown_F(i, j); S(i, j + 3) = Brown_H(i, j);
            S(i + 3, j) = Neel_F(i, j); S(i + 3, j + 3) = Neel_H(i, j);
        }
        return S;
    }
    // .inl:179-219
    Dep getDrift(const Dep& yi) const {
        const V3<T> ni = head(yi), ei = tail(yi);
        const T cF_2 = cF * cF;
        const T PreH_2 = DN * DN;
        V3<T> brown, neel;
        if (simple) {
            brown = ni * (-cF_2);
            neel = ei * (-((a_ * a_ + b_ * b_) * PreH_2));
        } else {
            const T& c = c_;
            const T d = c * MagneticMoment;
            const T bpd = b_ + d;
            const V3<T> nixei = cross(ni, ei);
            const V3<T> nee = ni * dot(ei, ei);  // (ni*ei^T)*ei
            brown = ni * (-cF_2) + ((d * a_) * nixei - (T(0.5) * d * d) * (nee - ni)) * PreH_2;
            neel = ei * (-(cF_2 + (a_ * a_ + bpd * bpd) * PreH_2));
        }
        Dep r; for (int i = 0; i < 3; ++i) { r[i] = brown[i]; r[3 + i] = neel[i]; } return r;
    }
    // .h:119-128: both Jacobians are identically zero in the reference
    Mat<T, 6, 6> getJacobiDeterministic(const Dep&, const V3<T>&, const T&) const { return Mat<T, 6, 6>::zero(); }
    Mat<T, 6, 6> getJacobiStochastic(const Vec<T, 6>&) const { return Mat<T, 6, 6>::zero(); }
    Vec<T, OUT> calculateOutputResult(const Dep& yi) const { return yi; }
    // BrownAndNeelRelaxation.h:168-172: n and m separately
    void normalize(Dep& yi) const {
        for (int h = 0; h < 6; h += 3) {
            const T n2 = yi[h] * yi[h] + yi[h + 1] * yi[h + 1] + yi[h + 2] * yi[h + 2];
            if (n2 > T(0.0)) { const T n = sqrt(n2); for (int k = 0; k < 3; ++k) yi[h + k] = yi[h + k] / n; }
        }
    }
};

}  // namespace orc
