// Generated by gen_moments.py -- do not edit.
#pragma once
namespace lbf {
// ---- D2Q9 ----
struct D2Q9_moments {
    static constexpr int Q = 9;
    static constexpr int rownorm2[9] = {9, 36, 36, 6, 12, 6, 12, 4, 4};
};
template <class R>
__device__ __forceinline__ void forward_d2q9(const R (&f)[9], R (&m)[9])
{
    const R a0 = f[1] + f[3], b0 = f[1] - f[3];
    const R a1 = f[2] + f[4], b1 = f[2] - f[4];
    const R a2 = f[5] + f[7], b2 = f[5] - f[7];
    const R a3 = f[6] + f[8], b3 = f[6] - f[8];
    m[0] = f[0] + a0 + a1 + a2 + a3;
    m[1] = -R(4) * f[0] - a0 - a1 + R(2) * a2 + R(2) * a3;
    m[2] = R(4) * f[0] - R(2) * a0 - R(2) * a1 + a2 + a3;
    m[3] = b0 + b2 - b3;
    m[4] = -R(2) * b0 + b2 - b3;
    m[5] = b1 + b2 + b3;
    m[6] = -R(2) * b1 + b2 + b3;
    m[7] = a0 - a1;
    m[8] = a2 - a3;
}
template <class R>
__device__ __forceinline__ void inverse_add_d2q9(const R (&c)[9], R (&f)[9])
{
    f[0] += c[0] - R(4) * c[1] + R(4) * c[2];
    { const R ev = c[0] - c[1] - R(2) * c[2] + c[7], od = c[3] - R(2) * c[4];
      f[1] += ev + od; f[3] += ev - od; }
    { const R ev = c[0] - c[1] - R(2) * c[2] - c[7], od = c[5] - R(2) * c[6];
      f[2] += ev + od; f[4] += ev - od; }
    { const R ev = c[0] + R(2) * c[1] + c[2] + c[8], od = c[3] + c[4] + c[5] + c[6];
      f[5] += ev + od; f[7] += ev - od; }
    { const R ev = c[0] + R(2) * c[1] + c[2] - c[8], od = -c[3] - c[4] + c[5] + c[6];
      f[6] += ev + od; f[8] += ev - od; }
}
// Equilibrium moments; rho may be the density deviation (shifted storage).
template <class R>
__device__ __forceinline__ R meq_d2q9(int k, R rho, R rho0, const R (&u)[3], const R (&uu)[6])
{
    // uu = {ux*ux, uy*uy, uz*uz, ux*uy, ux*uz, uy*uz}
    switch (k) {
    case 0: return rho + rho0 * (R(0));
    case 1: return R(-2) * rho + rho0 * (R(3) * uu[0] + R(3) * uu[1]);
    case 2: return rho + rho0 * (-R(3) * uu[0] - R(3) * uu[1]);
    case 3: return rho0 * (u[0]);
    case 4: return rho0 * (-u[0]);
    case 5: return rho0 * (u[1]);
    case 6: return rho0 * (-u[1]);
    case 7: return rho0 * (uu[0] - uu[1]);
    case 8: return rho0 * (uu[3]);
    default: return R(0);
    }
}
// Guo source moments; uF[a][b] = u_a F_b, uf = u.F.
template <class R>
__device__ __forceinline__ R msrc_d2q9(int k, const R (&F)[3], const R (&uF)[3][3], R uf)
{
    switch (k) {
    case 0: return R(3) * uF[0][0] + R(3) * uF[1][1] - R(3) * uf;
    case 1: return R(6) * uf;
    case 2: return -R(3) * uF[0][0] - R(3) * uF[1][1] - R(3) * uf;
    case 3: return F[0];
    case 4: return -F[0];
    case 5: return F[1];
    case 6: return -F[1];
    case 7: return R(2) * uF[0][0] - R(2) * uF[1][1];
    case 8: return uF[0][1] + uF[1][0];
    default: return R(0);
    }
}
// ---- D3Q19 ----
struct D3Q19_moments {
    static constexpr int Q = 19;
    static constexpr int rownorm2[19] = {19, 2394, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8};
};
template <class R>
__device__ __forceinline__ void forward_d3q19(const R (&f)[19], R (&m)[19])
{
    const R a0 = f[1] + f[2], b0 = f[1] - f[2];
    const R a1 = f[3] + f[4], b1 = f[3] - f[4];
    const R a2 = f[5] + f[6], b2 = f[5] - f[6];
    const R a3 = f[7] + f[10], b3 = f[7] - f[10];
    const R a4 = f[8] + f[9], b4 = f[8] - f[9];
    const R a5 = f[11] + f[14], b5 = f[11] - f[14];
    const R a6 = f[12] + f[13], b6 = f[12] - f[13];
    const R a7 = f[15] + f[18], b7 = f[15] - f[18];
    const R a8 = f[16] + f[17], b8 = f[16] - f[17];
    m[0] = f[0] + a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7 + a8;
    m[1] = -R(30) * f[0] - R(11) * a0 - R(11) * a1 - R(11) * a2 + R(8) * a3 + R(8) * a4 + R(8) * a5 + R(8) * a6 + R(8) * a7 + R(8) * a8;
    m[2] = R(12) * f[0] - R(4) * a0 - R(4) * a1 - R(4) * a2 + a3 + a4 + a5 + a6 + a7 + a8;
    m[3] = b0 + b3 - b4 + b5 - b6;
    m[4] = -R(4) * b0 + b3 - b4 + b5 - b6;
    m[5] = b1 + b3 + b4 + b7 - b8;
    m[6] = -R(4) * b1 + b3 + b4 + b7 - b8;
    m[7] = b2 + b5 + b6 + b7 + b8;
    m[8] = -R(4) * b2 + b5 + b6 + b7 + b8;
    m[9] = R(2) * a0 - a1 - a2 + a3 + a4 + a5 + a6 - R(2) * a7 - R(2) * a8;
    m[10] = -R(4) * a0 + R(2) * a1 + R(2) * a2 + a3 + a4 + a5 + a6 - R(2) * a7 - R(2) * a8;
    m[11] = a1 - a2 + a3 + a4 - a5 - a6;
    m[12] = -R(2) * a1 + R(2) * a2 + a3 + a4 - a5 - a6;
    m[13] = a3 - a4;
    m[14] = a7 - a8;
    m[15] = a5 - a6;
    m[16] = b3 - b4 - b5 + b6;
    m[17] = -b3 - b4 + b7 - b8;
    m[18] = b5 + b6 - b7 - b8;
}
template <class R>
__device__ __forceinline__ void inverse_add_d3q19(const R (&c)[19], R (&f)[19])
{
    f[0] += c[0] - R(30) * c[1] + R(12) * c[2];
    { const R ev = c[0] - R(11) * c[1] - R(4) * c[2] + R(2) * c[9] - R(4) * c[10], od = c[3] - R(4) * c[4];
      f[1] += ev + od; f[2] += ev - od; }
    { const R ev = c[0] - R(11) * c[1] - R(4) * c[2] - c[9] + R(2) * c[10] + c[11] - R(2) * c[12], od = c[5] - R(4) * c[6];
      f[3] += ev + od; f[4] += ev - od; }
    { const R ev = c[0] - R(11) * c[1] - R(4) * c[2] - c[9] + R(2) * c[10] - c[11] + R(2) * c[12], od = c[7] - R(4) * c[8];
      f[5] += ev + od; f[6] += ev - od; }
    { const R ev = c[0] + R(8) * c[1] + c[2] + c[9] + c[10] + c[11] + c[12] + c[13], od = c[3] + c[4] + c[5] + c[6] + c[16] - c[17];
      f[7] += ev + od; f[10] += ev - od; }
    { const R ev = c[0] + R(8) * c[1] + c[2] + c[9] + c[10] + c[11] + c[12] - c[13], od = -c[3] - c[4] + c[5] + c[6] - c[16] - c[17];
      f[8] += ev + od; f[9] += ev - od; }
    { const R ev = c[0] + R(8) * c[1] + c[2] + c[9] + c[10] - c[11] - c[12] + c[15], od = c[3] + c[4] + c[7] + c[8] - c[16] + c[18];
      f[11] += ev + od; f[14] += ev - od; }
    { const R ev = c[0] + R(8) * c[1] + c[2] + c[9] + c[10] - c[11] - c[12] - c[15], od = -c[3] - c[4] + c[7] + c[8] + c[16] + c[18];
      f[12] += ev + od; f[13] += ev - od; }
    { const R ev = c[0] + R(8) * c[1] + c[2] - R(2) * c[9] - R(2) * c[10] + c[14], od = c[5] + c[6] + c[7] + c[8] + c[17] - c[18];
      f[15] += ev + od; f[18] += ev - od; }
    { const R ev = c[0] + R(8) * c[1] + c[2] - R(2) * c[9] - R(2) * c[10] - c[14], od = -c[5] - c[6] + c[7] + c[8] - c[17] - c[18];
      f[16] += ev + od; f[17] += ev - od; }
}
// Equilibrium moments; rho may be the density deviation (shifted storage).
template <class R>
__device__ __forceinline__ R meq_d3q19(int k, R rho, R rho0, const R (&u)[3], const R (&uu)[6])
{
    // uu = {ux*ux, uy*uy, uz*uz, ux*uy, ux*uz, uy*uz}
    switch (k) {
    case 0: return rho + rho0 * (R(0));
    case 1: return R(-11) * rho + rho0 * (R(19) * uu[0] + R(19) * uu[1] + R(19) * uu[2]);
    case 2: return R(3) * rho + rho0 * (-R(5.5) * uu[0] - R(5.5) * uu[1] - R(5.5) * uu[2]);
    case 3: return rho0 * (u[0]);
    case 4: return rho0 * (-R(0.6666666666666666) * u[0]);
    case 5: return rho0 * (u[1]);
    case 6: return rho0 * (-R(0.6666666666666666) * u[1]);
    case 7: return rho0 * (u[2]);
    case 8: return rho0 * (-R(0.6666666666666666) * u[2]);
    case 9: return rho0 * (R(2) * uu[0] - uu[1] - uu[2]);
    case 10: return rho0 * (-uu[0] + R(0.5) * uu[1] + R(0.5) * uu[2]);
    case 11: return rho0 * (uu[1] - uu[2]);
    case 12: return rho0 * (-R(0.5) * uu[1] + R(0.5) * uu[2]);
    case 13: return rho0 * (uu[3]);
    case 14: return rho0 * (uu[5]);
    case 15: return rho0 * (uu[4]);
    case 16: return rho0 * (R(0));
    case 17: return rho0 * (R(0));
    case 18: return rho0 * (R(0));
    default: return R(0);
    }
}
// Guo source moments; uF[a][b] = u_a F_b, uf = u.F.
template <class R>
__device__ __forceinline__ R msrc_d3q19(int k, const R (&F)[3], const R (&uF)[3][3], R uf)
{
    switch (k) {
    case 0: return R(3) * uF[0][0] + R(3) * uF[1][1] + R(3) * uF[2][2] - R(3) * uf;
    case 1: return R(5) * uF[0][0] + R(5) * uF[1][1] + R(5) * uF[2][2] + R(33) * uf;
    case 2: return -R(2) * uF[0][0] - R(2) * uF[1][1] - R(2) * uF[2][2] - R(9) * uf;
    case 3: return F[0];
    case 4: return -R(0.6666666666666666) * F[0];
    case 5: return F[1];
    case 6: return -R(0.6666666666666666) * F[1];
    case 7: return F[2];
    case 8: return -R(0.6666666666666666) * F[2];
    case 9: return R(4) * uF[0][0] - R(2) * uF[1][1] - R(2) * uF[2][2];
    case 10: return -R(2) * uF[0][0] + uF[1][1] + uF[2][2];
    case 11: return R(2) * uF[1][1] - R(2) * uF[2][2];
    case 12: return -uF[1][1] + uF[2][2];
    case 13: return uF[0][1] + uF[1][0];
    case 14: return uF[1][2] + uF[2][1];
    case 15: return uF[0][2] + uF[2][0];
    case 16: return R(0);
    case 17: return R(0);
    case 18: return R(0);
    default: return R(0);
    }
}
}  // namespace lbf
