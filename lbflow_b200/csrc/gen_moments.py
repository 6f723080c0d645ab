#!/usr/bin/env python3
"""Generate moments_gen.cuh: straight-line MRT moment code for D2Q9 and D3Q19.

The MRT collision of LBFlow (solver/src/lbm/scsp.cpp:411-464 and
colorfluid.cpp:360-387) relaxes the moments m = M f of the populations with
the transform M of solver/src/lbm/simulator.cpp:162-197.  The engine evaluates
it in moment space:

  m      = M f                      (forward, opposite pairs folded first)
  meq_k  = A_k rho + rho0 (3 B_k.u + 4.5 u.C_k.u - 1.5 A_k |u|^2)
  msrc_k = 3 B_k.F - 3 A_k (u.F) + 9 u.C_k.F      (Guo source moments)
  f     += M^T c,   c_k = (s_k (meq_k - m_k) + (1 - s_k/2) msrc_k) / |M_k|^2

with A_k = sum_q M_kq w_q, B_ka = sum_q M_kq w_q e_qa and
C_kab = sum_q M_kq w_q e_qa e_qb evaluated here in exact rational arithmetic.
Rows are emitted only with their non-zero terms, so the compiler sees plain
adds and multiplies by literal constants.  Run from this directory:

    python gen_moments.py > moments_gen.cuh
"""
from fractions import Fraction as Fr

# Reference q ordering; vectors written as (x, y, z).
D2Q9 = dict(
    name='d2q9', D=2,
    e=[(0, 0, 0), (1, 0, 0), (0, 1, 0), (-1, 0, 0), (0, -1, 0),
       (1, 1, 0), (-1, 1, 0), (-1, -1, 0), (1, -1, 0)],
    w=[Fr(16, 36)] + [Fr(4, 36)] * 4 + [Fr(1, 36)] * 4,
    M=[[1, 1, 1, 1, 1, 1, 1, 1, 1],
       [-4, -1, -1, -1, -1, 2, 2, 2, 2],
       [4, -2, -2, -2, -2, 1, 1, 1, 1],
       [0, 1, 0, -1, 0, 1, -1, -1, 1],
       [0, -2, 0, 2, 0, 1, -1, -1, 1],
       [0, 0, 1, 0, -1, 1, 1, -1, -1],
       [0, 0, -2, 0, 2, 1, 1, -1, -1],
       [0, 1, -1, 1, -1, 0, 0, 0, 0],
       [0, 0, 0, 0, 0, 1, -1, 1, -1]],
)
D3Q19 = dict(
    name='d3q19', D=3,
    e=[(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
       (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0),
       (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1),
       (0, 1, 1), (0, -1, 1), (0, 1, -1), (0, -1, -1)],
    w=[Fr(12, 36)] + [Fr(2, 36)] * 6 + [Fr(1, 36)] * 12,
    M=[[1] * 19,
       [-30] + [-11] * 6 + [8] * 12,
       [12] + [-4] * 6 + [1] * 12,
       [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
       [0, -4, 4, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
       [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1],
       [0, 0, 0, -4, 4, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1],
       [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1],
       [0, 0, 0, 0, 0, -4, 4, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1],
       [0, 2, 2, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2],
       [0, -4, -4, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, -2, -2, -2, -2],
       [0, 0, 0, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0],
       [0, 0, 0, -2, -2, 2, 2, 1, 1, 1, 1, -1, -1, -1, -1, 0, 0, 0, 0],
       [0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 0, 0, 0, 0],
       [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1],
       [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0],
       [0, 0, 0, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1, 0, 0, 0, 0],
       [0, 0, 0, 0, 0, 0, 0, -1, -1, 1, 1, 0, 0, 0, 0, 1, -1, 1, -1],
       [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, -1, -1, -1, -1, 1, 1]],
)


def lit(x):
    v = float(x)
    if v == int(v) and abs(v) < 1e15:
        return f'R({int(v)})'
    return f'R({v!r})'


def lin(terms):
    """Sum of (coef, expr) terms as a C expression."""
    out = ''
    for c, ex in terms:
        if c == 0:
            continue
        if c == 1:
            t = ex
            sign = '+'
        elif c == -1:
            t = ex
            sign = '-'
        else:
            t = f'{lit(abs(c))} * {ex}'
            sign = '+' if c > 0 else '-'
        if not out:
            out = t if sign == '+' else f'-{t}'
        else:
            out += f' {sign} {t}'
    return out or 'R(0)'


def gen(L):
    e, w, M, D = L['e'], L['w'], L['M'], L['D']
    Q = len(e)
    op = [next(r for r in range(Q) if all(e[r][a] == -e[q][a] for a in range(3))) for q in range(Q)]
    pairs = []
    for q in range(1, Q):
        if q < op[q]:
            pairs.append(q)
    parity = []
    for k in range(Q):
        even = all(M[k][q] == M[k][op[q]] for q in range(1, Q))
        odd = all(M[k][q] == -M[k][op[q]] for q in range(1, Q)) and M[k][0] == 0
        assert even or odd
        parity.append(1 if even else -1)
    A = [sum(M[k][q] * w[q] for q in range(Q)) for k in range(Q)]
    B = [[sum(M[k][q] * w[q] * e[q][a] for q in range(Q)) for a in range(3)] for k in range(Q)]
    C = [[[sum(M[k][q] * w[q] * e[q][a] * e[q][b] for q in range(Q)) for b in range(3)]
          for a in range(3)] for k in range(Q)]
    n2 = [sum(M[k][q] ** 2 for q in range(Q)) for k in range(Q)]
    name = L['name']
    o = []
    o.append(f'// ---- {name.upper()} ----')
    o.append(f'struct {name.upper()}_moments {{')
    o.append(f'    static constexpr int Q = {Q};')
    o.append(f'    static constexpr int rownorm2[{Q}] = {{{", ".join(map(str, n2))}}};')
    o.append('};')
    # forward
    o.append('template <class R>')
    o.append(f'__device__ __forceinline__ void forward_{name}(const R (&f)[{Q}], R (&m)[{Q}])')
    o.append('{')
    for i, q in enumerate(pairs):
        o.append(f'    const R a{i} = f[{q}] + f[{op[q]}], b{i} = f[{q}] - f[{op[q]}];')
    for k in range(Q):
        if parity[k] > 0:
            terms = [(M[k][0], 'f[0]')] + [(M[k][q], f'a{i}') for i, q in enumerate(pairs)]
        else:
            terms = [(M[k][q], f'b{i}') for i, q in enumerate(pairs)]
        o.append(f'    m[{k}] = {lin(terms)};')
    o.append('}')
    # inverse
    o.append('template <class R>')
    o.append(f'__device__ __forceinline__ void inverse_add_{name}(const R (&c)[{Q}], R (&f)[{Q}])')
    o.append('{')
    o.append(f'    f[0] += {lin([(M[k][0], f"c[{k}]") for k in range(Q) if parity[k] > 0])};')
    for i, q in enumerate(pairs):
        ev = lin([(M[k][q], f'c[{k}]') for k in range(Q) if parity[k] > 0])
        od = lin([(M[k][q], f'c[{k}]') for k in range(Q) if parity[k] < 0])
        o.append(f'    {{ const R ev = {ev}, od = {od};')
        o.append(f'      f[{q}] += ev + od; f[{op[q]}] += ev - od; }}')
    o.append('}')
    # equilibrium moments
    o.append('// Equilibrium moments; rho may be the density deviation (shifted storage).')
    o.append('template <class R>')
    o.append(f'__device__ __forceinline__ R meq_{name}(int k, R rho, R rho0, const R (&u)[3], const R (&uu)[6])')
    o.append('{')
    o.append('    // uu = {ux*ux, uy*uy, uz*uz, ux*uy, ux*uz, uy*uz}')
    o.append('    switch (k) {')
    idx = {(0, 0): 0, (1, 1): 1, (2, 2): 2, (0, 1): 3, (0, 2): 4, (1, 2): 5}
    for k in range(Q):
        lt = [(3 * B[k][a], f'u[{a}]') for a in range(D)]
        qt = {}
        for a in range(D):
            for b in range(D):
                c = Fr(9, 2) * C[k][a][b] - (Fr(3, 2) * A[k] if a == b else 0)
                key = idx[(min(a, b), max(a, b))]
                qt[key] = qt.get(key, 0) + c
        terms = lt + [(qt[k2], f'uu[{k2}]') for k2 in sorted(qt)]
        inner = lin(terms)
        pre = '' if A[k] == 0 else (f'{lit(A[k])} * rho + ' if A[k] != 1 else 'rho + ')
        o.append(f'    case {k}: return {pre}rho0 * ({inner});')
    o.append('    default: return R(0);')
    o.append('    }')
    o.append('}')
    # source moments
    o.append('// Guo source moments; uF[a][b] = u_a F_b, uf = u.F.')
    o.append('template <class R>')
    o.append(f'__device__ __forceinline__ R msrc_{name}(int k, const R (&F)[3], const R (&uF)[3][3], R uf)')
    o.append('{')
    o.append('    switch (k) {')
    for k in range(Q):
        terms = [(3 * B[k][a], f'F[{a}]') for a in range(D)]
        for a in range(D):
            for b in range(D):
                terms.append((9 * C[k][a][b], f'uF[{a}][{b}]'))
        if A[k] != 0:
            terms.append((-3 * A[k], 'uf'))
        o.append(f'    case {k}: return {lin(terms)};')
    o.append('    default: return R(0);')
    o.append('    }')
    o.append('}')
    return '\n'.join(o)


def main():
    print('// Generated by gen_moments.py -- do not edit.')
    print('#pragma once')
    print('namespace lbf {')
    print(gen(D2Q9))
    print(gen(D3Q19))
    print('}  // namespace lbf')


if __name__ == '__main__':
    main()
