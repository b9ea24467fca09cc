"""Generator of the per-class shell-quartet recursions (CUDA device code).

For a quartet class (la lb | lc ld) with la <= lb, lc <= ld the emitted code
follows the Head-Gordon-Pople scheme the reference uses
(src/t4c_electron_repulsion/ElectronRepulsionRec*.hpp):

1. per primitive quartet, Obara-Saika vertical recursion on centres B and D
   producing [0 e | 0 f]^(0) for |e| in [lb, la+lb], |f| in [ld, lc+ld]
   (reference: ElectronRepulsionPrimRec*.cpp);
2. sum over primitive quartets (reference: t2cfunc::reduce);
3. ket horizontal recursion |c+1_i, d) = |c, d+1_i) + (D_i - C_i)|c, d)
   (reference: ElectronRepulsionContrRecXX*.cpp);
4. ket Cartesian -> spherical (t4cfunc::ket_transform);
5. bra horizontal recursion (a+1_i, b| = (a, b+1_i| + (B_i - A_i)(a, b|
   on the half-spherical data (ElectronRepulsionContrRec*XX.cpp);
6. bra Cartesian -> spherical (t4cfunc::bra_transform).

The recursion graph is built here by demand-driven expansion from the
targets, so only the intermediates a class needs are emitted, as straight-line
code (registers) that the compiler schedules.  Spherical factors are the real
solid harmonics normalised with the reference's primitive normalisation
(src/general/SphericalMomentum.hpp conventions: m = -l..l, p = (y, z, x)).

Usage: python gen_eri.py OUTDIR [LMAX]
"""

import math
import re
import sys
from pathlib import Path

# ----------------------------------------------------------------- components

def cart_list(l):
    """Lexicographic Cartesian components of angular momentum l (xx, xy, xz, ...)."""
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def ncart(l):
    return (l + 1) * (l + 2) // 2


def _binom(n, k):
    return math.comb(n, k) if 0 <= k <= n else 0


_LNORM = {0: 1.0, 1: 2.0, 2: 2.0 / math.sqrt(3.0), 3: 4.0 / math.sqrt(15.0), 4: 2.0 / math.sqrt(105.0)}


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def sph_coefficients(l):
    """rows m = -l..l, columns lexicographic Cartesian components."""
    carts = cart_list(l)
    idx = {c: i for i, c in enumerate(carts)}
    rows = []
    for m in range(-l, l + 1):
        am = abs(m)
        c = [0.0] * len(carts)
        vm2 = 1 if m < 0 else 0  # 2*vm
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                v2 = vm2
                while v2 <= 2 * ((am - vm2) // 2) + vm2 and v2 <= am:
                    sgn = -1.0 if ((2 * t + v2 - vm2) // 2) % 2 else 1.0
                    coef = sgn * 0.25 ** t * _binom(l, t) * _binom(l - t, am + t) * _binom(t, u) * _binom(am, v2)
                    px, py, pz = 2 * t + am - 2 * u - v2, 2 * u + v2, l - 2 * t - am
                    if px >= 0 and py >= 0 and pz >= 0:
                        c[idx[(px, py, pz)]] += coef
                    v2 += 2
        nrm = 0.0
        for i, ci in enumerate(carts):
            for j, cj in enumerate(carts):
                s = [ci[k] + cj[k] for k in range(3)]
                if any(v % 2 for v in s):
                    continue
                nrm += c[i] * c[j] * _dfact(s[0] - 1) * _dfact(s[1] - 1) * _dfact(s[2] - 1)
        scale = 1.0 / math.sqrt(nrm * _LNORM[l] ** 2 / 4.0 ** l)
        rows.append([v * scale for v in c])
    return rows


def sub1(c, i):
    v = list(c)
    v[i] -= 1
    return tuple(v)


def add1(c, i):
    v = list(c)
    v[i] += 1
    return tuple(v)


def pick_axis(c):
    """Axis used to lower a component: the first axis (x, y, z) with the largest exponent."""
    best = max(c)
    for i in range(3):
        if c[i] == best and best > 0:
            return i
    raise ValueError(c)


# ----------------------------------------------------------------- VRR graph

class VRR:
    """Demand-driven OS vertical recursion for [0 e | 0 f]^(m)."""

    def __init__(self):
        self.nodes = {}   # key -> (expr terms)
        self.order = []

    def need(self, e, f, m):
        key = (e, f, m)
        if key in self.nodes:
            return key
        terms = []
        if sum(f) > 0:
            i = pick_axis(f)
            f1 = sub1(f, i)
            terms.append(('QD', i, self.need(e, f1, m)))
            terms.append(('WQ', i, self.need(e, f1, m + 1)))
            if f1[i] > 0:
                f2 = sub1(f1, i)
                terms.append(('F2', f1[i], self.need(e, f2, m), self.need(e, f2, m + 1)))
            if e[i] > 0:
                terms.append(('EZH', e[i], self.need(sub1(e, i), f1, m + 1)))
        elif sum(e) > 0:
            i = pick_axis(e)
            e1 = sub1(e, i)
            terms.append(('PB', i, self.need(e1, f, m)))
            terms.append(('WP', i, self.need(e1, f, m + 1)))
            if e1[i] > 0:
                e2 = sub1(e1, i)
                terms.append(('E2', e1[i], self.need(e2, f, m), self.need(e2, f, m + 1)))
        else:
            terms.append(('BASE', m))
        self.nodes[key] = terms
        self.order.append(key)
        return key


# ----------------------------------------------------------------- emitter

AX = 'xyz'


class ClassGen:
    def __init__(self, la, lb, lc, ld):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.L = la + lb + lc + ld
        self.e_targets = [c for l in range(lb, la + lb + 1) for c in cart_list(l)]
        self.f_targets = [c for l in range(ld, lc + ld + 1) for c in cart_list(l)]
        self.vrr = VRR()
        for e in self.e_targets:
            for f in self.f_targets:
                self.vrr.need(e, f, 0)
        self.names = {}
        for k, key in enumerate(self.vrr.order):
            self.names[key] = 'v%d' % k

    def stats(self):
        return dict(vrr=len(self.vrr.order), acc=len(self.e_targets) * len(self.f_targets))

    def _vrr_expr(self, key):
        terms = self.vrr.nodes[key]
        n = self.names
        out = []
        for t in terms:
            if t[0] == 'BASE':
                return 'F[%d]' % t[1]
            if t[0] == 'QD':
                out.append('QD%s * %s' % (AX[t[1]], n[t[2]]))
            elif t[0] == 'WQ':
                out.append('WQ%s * %s' % (AX[t[1]], n[t[2]]))
            elif t[0] == 'PB':
                out.append('PB%s * %s' % (AX[t[1]], n[t[2]]))
            elif t[0] == 'WP':
                out.append('WP%s * %s' % (AX[t[1]], n[t[2]]))
            elif t[0] == 'F2':
                out.append('%s * hie * (%s - rh * %s)' % (_num(t[1]), n[t[2]], n[t[3]]))
            elif t[0] == 'E2':
                out.append('%s * hiz * (%s - rz * %s)' % (_num(t[1]), n[t[2]], n[t[3]]))
            elif t[0] == 'EZH':
                out.append('%s * hizh * %s' % (_num(t[1]), n[t[2]]))
        return ' + '.join(out)

    def closure(self, keys):
        """VRR nodes the given nodes depend on (themselves included), in the
        emission order."""
        seen, stack = set(), list(keys)
        while stack:
            k = stack.pop()
            if k in seen:
                continue
            seen.add(k)
            for term in self.vrr.nodes[k]:
                for x in term[2:]:
                    if isinstance(x, tuple):
                        stack.append(x)
        return [k for k in self.vrr.order if k in seen]

    def emit(self, real='double', parts=1):
        """parts > 1: the accumulator rows (bra Cartesian targets e) are
        evaluated in `parts` groups, each with its own primitive loop over only
        the recursion nodes its rows need, and ket-transformed into the
        half-transformed values h_e_k_l before the next group starts, so that
        only one group's accumulators are live at a time (for classes whose
        contracted buffer does not fit the registers)."""
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        L = self.L
        na, nb, nc, nd = 2 * la + 1, 2 * lb + 1, 2 * lc + 1, 2 * ld + 1
        nsph = na * nb * nc * nd
        e_t, f_t = self.e_targets, self.f_targets
        lines = []
        w = lines.append
        w('// class (%d %d | %d %d): %d VRR nodes, %d contracted accumulators, %d spherical outputs'
          % (la, lb, lc, ld, len(self.vrr.order), len(e_t) * len(f_t), nsph))
        w('template <> struct EriClass<%d, %d, %d, %d> {' % (la, lb, lc, ld))
        w('    static constexpr int NSPH = %d;' % nsph)
        method_start = len(lines)
        w('    template <class BraT, class KetT>')
        w('    __device__ __forceinline__ static void compute(const BraT& bra, const KetT& ket, const double* __restrict__ btab,')
        w('                                                   const double om2, double* __restrict__ out)')
        w('    {')
        groups = [list(range(len(e_t)))[r::parts] for r in range(parts)]
        if parts > 1:
            for ie in range(len(e_t)):
                for k in range(nc):
                    for l in range(nd):
                        w('        double h_%d_%d_%d;' % (ie, k, l))
        w('        const int kb = bra.nprim(), kk = ket.nprim();')
        for group in groups:
            self._emit_group(w, group, parts > 1)
        if parts > 1:
            w('        const double BAx = bra.abx(), BAy = bra.aby(), BAz = bra.abz();')
            w('        (void)BAx; (void)BAy; (void)BAz;')
        self._emit_bra(w)
        if parts == 1:
            w('        }')
        w('    }')
        body = lines[method_start:]
        lines.extend(to_f32(body))
        w('};')
        return '\n'.join(lines)

    def _emit_group(self, w, group, store):
        """Primitive loop and ket transform of the accumulator rows `group`
        (indices into e_targets); store: assign to the function-scope h_e_k_l
        (grouped emission) instead of declaring them."""
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        L = self.L
        nc, nd = 2 * lc + 1, 2 * ld + 1
        e_t, f_t = self.e_targets, self.f_targets
        w('        {')
        for ie in group:
            for jf in range(len(f_t)):
                w('        double c_%d_%d = 0.0;' % (ie, jf))
        # ket primitives outer: the ket data is per lane (loaded once per ket
        # primitive), the bra data is warp-uniform (broadcast loads)
        w('        for (int pk = 0; pk < kk; pk++) {')
        w('            const double eta = ket.zeta(pk), hie = ket.hiz(pk), kcd = ket.kfac(pk);')
        w('            const double QDx = ket.pbx(pk), QDy = ket.pby(pk), QDz = ket.pbz(pk);')
        w('            const double Qx = ket.px(pk), Qy = ket.py(pk), Qz = ket.pz(pk);')
        w('            for (int pb = 0; pb < kb; pb++) {')
        w('                const double zeta = bra.zeta(pb), hiz = bra.hiz(pb), kab = bra.kfac(pb);')
        w('                const double PBx = bra.pbx(pb), PBy = bra.pby(pb), PBz = bra.pbz(pb);')
        w('                const double PQx = bra.px(pb) - Qx, PQy = bra.py(pb) - Qy, PQz = bra.pz(pb) - Qz;')
        w('                const double r = rsqrt(zeta + eta);')
        w('                const double inv = r * r;')
        w('                const double rz = eta * inv, rh = zeta * inv;')
        w('                const double rho = zeta * rz;')
        w('                const double hizh = 0.5 * inv;')
        w('                const double WPx = -rz * PQx, WPy = -rz * PQy, WPz = -rz * PQz;')
        w('                const double WQx = rh * PQx, WQy = rh * PQy, WQz = rh * PQz;')
        w('                const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);')
        w('                double F[%d];' % (L + 1))
        # F_m scaled by the primitive prefactor inside the Boys evaluation;
        # erf-attenuated operator: F_m(T) -> s^(2m+1) F_m(s^2 T), s^2 = om2 / (om2 + rho)
        w('                double Tb = T;')
        w('                double sc = kab * kcd * r;')
        w('                double s2 = 1.0;')
        w('                if (om2 > 0.0) {')
        w('                    s2 = om2 / (om2 + rho);')
        w('                    Tb = T * s2;')
        w('                    sc *= sqrt(s2);')
        w('                }')
        w('                boys_scaled<%d>(Tb, sc, F, btab);' % L)
        if L > 0:
            w('                if (om2 > 0.0) {')
            w('                    double sm = s2;')
            w('                    #pragma unroll')
            w('                    for (int m = 1; m <= %d; m++) {' % L)
            w('                        F[m] *= sm;')
            w('                        sm *= s2;')
            w('                    }')
            w('                }')
        w('                (void)WPx; (void)WPy; (void)WPz; (void)WQx; (void)WQy; (void)WQz;')
        w('                (void)QDx; (void)QDy; (void)QDz; (void)PBx; (void)PBy; (void)PBz;')
        w('                (void)hiz; (void)hie; (void)hizh; (void)rz; (void)rh;')
        needed = self.closure([(e_t[ie], f, 0) for ie in group for f in f_t])
        for key in needed:
            w('                const double %s = %s;' % (self.names[key], self._vrr_expr(key)))
        for ie in group:
            for jf, f in enumerate(f_t):
                w('                c_%d_%d += %s;' % (ie, jf, self.names[(e_t[ie], f, 0)]))
        w('            }')
        w('        }')
        # ---- ket HRR (per e target) then ket spherical
        w('        const double DCx = ket.abx(), DCy = ket.aby(), DCz = ket.abz();')
        w('        (void)DCx; (void)DCy; (void)DCz;')
        if not store:
            w('        const double BAx = bra.abx(), BAy = bra.aby(), BAz = bra.abz();')
            w('        (void)BAx; (void)BAy; (void)BAz;')
        f_index = {f: j for j, f in enumerate(f_t)}
        ket_nodes, ket_order = {}, []

        def need_ket(c, d):
            key = (c, d)
            if key in ket_nodes:
                return key
            if sum(c) == 0:
                ket_nodes[key] = ('F', f_index[d])
            else:
                i = pick_axis(c)
                c1 = sub1(c, i)
                ket_nodes[key] = ('H', i, need_ket(c1, add1(d, i)), need_ket(c1, d))
            ket_order.append(key)
            return key

        cc, dc = cart_list(lc), cart_list(ld)
        for c in cc:
            for d in dc:
                need_ket(c, d)
        sph_c, sph_d = sph_coefficients(lc), sph_coefficients(ld)
        # half-transformed buffer h[ie][k][l]
        for ie in group:
            names = {}
            for n_, key in enumerate(ket_order):
                node = ket_nodes[key]
                nm = 'k%d_%d' % (ie, n_)
                names[key] = nm
                if node[0] == 'F':
                    w('        const double %s = c_%d_%d;' % (nm, ie, node[1]))
                else:
                    w('        const double %s = %s + DC%s * %s;' % (nm, names[node[2]], AX[node[1]], names[node[3]]))
            for k in range(nc):
                for l in range(nd):
                    terms = []
                    for ic, c in enumerate(cc):
                        if sph_c[k][ic] == 0.0:
                            continue
                        for jd, d in enumerate(dc):
                            if sph_d[l][jd] == 0.0:
                                continue
                            terms.append('%s * %s' % (_num(sph_c[k][ic] * sph_d[l][jd]), names[(c, d)]))
                    w('        %sh_%d_%d_%d = %s;' % ('' if store else 'const double ', ie, k, l, ' + '.join(terms)))
        if not store:
            return  # single group: the bra part follows in the same scope
        w('        }')

    def _emit_bra(self, w):
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        na, nb, nc, nd = 2 * la + 1, 2 * lb + 1, 2 * lc + 1, 2 * ld + 1
        e_t = self.e_targets
        # ---- bra HRR per (k, l), then bra spherical
        e_index = {e: j for j, e in enumerate(e_t)}
        bra_nodes, bra_order = {}, []

        def need_bra(a, b):
            key = (a, b)
            if key in bra_nodes:
                return key
            if sum(a) == 0:
                bra_nodes[key] = ('E', e_index[b])
            else:
                i = pick_axis(a)
                a1 = sub1(a, i)
                bra_nodes[key] = ('H', i, need_bra(a1, add1(b, i)), need_bra(a1, b))
            bra_order.append(key)
            return key

        ac, bc = cart_list(la), cart_list(lb)
        for a in ac:
            for b in bc:
                need_bra(a, b)
        sph_a, sph_b = sph_coefficients(la), sph_coefficients(lb)
        for k in range(nc):
            for l in range(nd):
                names = {}
                for n_, key in enumerate(bra_order):
                    node = bra_nodes[key]
                    nm = 'b%d_%d_%d' % (k, l, n_)
                    names[key] = nm
                    if node[0] == 'E':
                        w('        const double %s = h_%d_%d_%d;' % (nm, node[1], k, l))
                    else:
                        w('        const double %s = %s + BA%s * %s;' % (nm, names[node[2]], AX[node[1]], names[node[3]]))
                for i in range(na):
                    for j in range(nb):
                        terms = []
                        for ia, a in enumerate(ac):
                            if sph_a[i][ia] == 0.0:
                                continue
                            for jb, b in enumerate(bc):
                                if sph_b[j][jb] == 0.0:
                                    continue
                                terms.append('%s * %s' % (_num(sph_a[i][ia] * sph_b[j][jb]), names[(a, b)]))
                        w('        out[%d] = %s;' % (((i * nb + j) * nc + k) * nd + l, ' + '.join(terms)))



    # --------------------------------------------------------- flop counts
    def flops(self):
        """Algorithmic FP64 operation counts of the recursion (1 per add or
        multiply): per primitive quartet the VRR graph (node-for-node the
        reference's ElectronRepulsionPrimRec* graph) plus one add per
        contracted accumulator; per contracted quartet the HRR nodes (2 each)
        and the spherical transforms (2 per nonzero factor)."""
        vrr = 0
        for key in self.vrr.order:
            terms = self.vrr.nodes[key]
            if terms[0][0] == 'BASE':
                continue
            for n_, t in enumerate(terms):
                cost = {'QD': 1, 'WQ': 1, 'PB': 1, 'WP': 1, 'F2': 4, 'E2': 4, 'EZH': 2}[t[0]]
                vrr += cost + (1 if n_ > 0 else 0)
        acc = len(self.e_targets) * len(self.f_targets)
        p = self.program()
        post = 0
        for op in p['post']:
            kind = op[0] >> 2
            if kind in (3, 4, 6):
                post += 2
        return vrr, acc, post

    # --------------------------------------------------------- interpreter
    def program(self):
        """Linear recursion program of the class (used for the operation counts).

        Slot 0 holds 0.0, slots 1..L+1 hold pref * F_m.  Ops (int4-quad + 2 doubles):
          kind 0/1  VRR bra/ket: S[t] = G1*S[a] + G2*S[b] + c1*H*(S[c] - R*S[d]) + c2*hizh*S[e]
          kind 2    accumulate:  S[t] += S[a]                       (per primitive quartet)
          kind 3/4  HRR ket/bra: S[t] = S[a] + G*S[b]               (G = D - C or B - A)
          kind 5    clear:       S[t] = 0
          kind 6    axpy:        S[t] += c1 * S[a]
        """
        L = self.L
        slot = {}
        nxt = [L + 2]

        def new():
            s = nxt[0]
            nxt[0] += 1
            return s

        vrr_ops = []
        for key in self.vrr.order:
            terms = self.vrr.nodes[key]
            if terms[0][0] == 'BASE':
                slot[key] = 1 + terms[0][1]
                continue
            t = new()
            slot[key] = t
            kind = 1 if terms[0][0] in ('QD', 'WQ') else 0
            axis = terms[0][1]
            a = slot[terms[0][2]]
            b = slot[terms[1][2]]
            c = d = e = 0
            c1 = c2 = 0.0
            for term in terms[2:]:
                if term[0] in ('F2', 'E2'):
                    c1 = float(term[1])
                    c, d = slot[term[2]], slot[term[3]]
                elif term[0] == 'EZH':
                    c2 = float(term[1])
                    e = slot[term[2]]
            vrr_ops.append((kind * 4 + axis, t, a, b, c, d, e, c1, c2))
        acc_slot = {}
        acc_ops = []
        for e in self.e_targets:
            for f in self.f_targets:
                s = new()
                acc_slot[(e, f)] = s
                acc_ops.append((2 * 4, s, slot[(e, f, 0)], 0, 0, 0, 0, 0.0, 0.0))
        post = []
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        nc_, nd_ = 2 * lc + 1, 2 * ld + 1
        na_, nb_ = 2 * la + 1, 2 * lb + 1
        cc, dc = cart_list(lc), cart_list(ld)
        ac, bc = cart_list(la), cart_list(lb)
        sph_c, sph_d = sph_coefficients(lc), sph_coefficients(ld)
        sph_a, sph_b = sph_coefficients(la), sph_coefficients(lb)
        # ket HRR per e target, then ket spherical -> h[e][k][l]
        hslot = {}
        for e in self.e_targets:
            knodes = {}

            def need_ket(c, d):
                if (c, d) in knodes:
                    return knodes[(c, d)]
                if sum(c) == 0:
                    knodes[(c, d)] = acc_slot[(e, d)]
                else:
                    i = pick_axis(c)
                    c1_ = sub1(c, i)
                    x = need_ket(c1_, add1(d, i))
                    y = need_ket(c1_, d)
                    t = new()
                    post.append((3 * 4 + i, t, x, y, 0, 0, 0, 0.0, 0.0))
                    knodes[(c, d)] = t
                return knodes[(c, d)]

            for c in cc:
                for d in dc:
                    need_ket(c, d)
            for k in range(nc_):
                for l in range(nd_):
                    t = new()
                    post.append((5 * 4, t, 0, 0, 0, 0, 0, 0.0, 0.0))
                    for ic, c in enumerate(cc):
                        for jd, d in enumerate(dc):
                            cf = sph_c[k][ic] * sph_d[l][jd]
                            if cf != 0.0:
                                post.append((6 * 4, t, knodes[(c, d)], 0, 0, 0, 0, cf, 0.0))
                    hslot[(e, k, l)] = t
        out_slots = [0] * (na_ * nb_ * nc_ * nd_)
        for k in range(nc_):
            for l in range(nd_):
                bnodes = {}

                def need_bra(a, b):
                    if (a, b) in bnodes:
                        return bnodes[(a, b)]
                    if sum(a) == 0:
                        bnodes[(a, b)] = hslot[(b, k, l)]
                    else:
                        i = pick_axis(a)
                        a1 = sub1(a, i)
                        x = need_bra(a1, add1(b, i))
                        y = need_bra(a1, b)
                        t = new()
                        post.append((4 * 4 + i, t, x, y, 0, 0, 0, 0.0, 0.0))
                        bnodes[(a, b)] = t
                    return bnodes[(a, b)]

                for a in ac:
                    for b in bc:
                        need_bra(a, b)
                for i in range(na_):
                    for j in range(nb_):
                        t = new()
                        post.append((5 * 4, t, 0, 0, 0, 0, 0, 0.0, 0.0))
                        for ia, a in enumerate(ac):
                            for jb, b in enumerate(bc):
                                cf = sph_a[i][ia] * sph_b[j][jb]
                                if cf != 0.0:
                                    post.append((6 * 4, t, bnodes[(a, b)], 0, 0, 0, 0, cf, 0.0))
                        out_slots[((i * nb_ + j) * nc_ + k) * nd_ + l] = t
        acc_first = min(acc_slot.values())
        return dict(nslots=nxt[0], vrr=vrr_ops, acc=acc_ops, post=post, out=out_slots,
                    acc_first=acc_first, nacc=len(acc_ops))

_FLOAT_LITERAL = re.compile(r'(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)(?![\w.])')


def to_f32(method_lines):
    """FP32 twin of the generated FP64 compute method (same recursion graph):
    compute_f32 with float intermediates, the float Boys table and float
    rsqrt; used for the small-bound quartets of the mixed-precision build."""
    out = []
    for line in method_lines:
        t = line.replace('static void compute(', 'static void compute_f32(')
        t = t.replace('const double* __restrict__ btab', 'const float* __restrict__ btab')
        t = t.replace('double* __restrict__ out', 'float* __restrict__ out')
        t = t.replace('const double ', 'const float ').replace('double c_', 'float c_').replace('double F[', 'float F[')
        t = t.replace('double h_', 'float h_')
        t = t.replace('boys_scaled<', 'boys_scaled_f<').replace('rsqrt(', 'rsqrtf(')
        t = re.sub(r'(?<![r\w])sqrt\(', 'sqrtf(', t)
        t = re.sub(r'\bdouble (Tb|sc|s2|sm)\b', r'float \1', t)
        if not t.lstrip().startswith('//'):
            t = _FLOAT_LITERAL.sub(lambda m: m.group(1) + 'f', t)
        out.append(t)
    return out


def _num(v):
    if isinstance(v, int):
        return '%d.0' % v
    if v == int(v) and abs(v) < 1e6:
        return '%d.0' % int(v)
    return repr(float(v))


# ----------------------------------------------------------------- classes

def pair_classes(lmax):
    return [(a, b) for a in range(lmax + 1) for b in range(a, lmax + 1)]


def pair_key(p):
    return (p[0] + p[1], p[1])


def quartet_classes(lmax):
    """Canonical classes: bra pair key >= ket pair key (the bra carries more
    angular momentum), each unordered pair of pair classes once."""
    pcs = sorted(pair_classes(lmax), key=pair_key)
    out = []
    for i, k in enumerate(pcs):
        for b in pcs[i:]:
            out.append((b[0], b[1], k[0], k[1]))
    return out


def class_name(c):
    return '%d%d%d%d' % c


def emit_class_file(cls, outdir):
    g = ClassGen(*cls)
    la, lb, lc, ld = cls
    nm = class_name(cls)
    body = []
    w = body.append
    w('// Generated by gen_eri.py -- do not edit.')
    w('#include "vlx_kernels.cuh"')
    w('namespace vlx {')
    w('template <> struct BlocksHint<%d, %d, %d, %d> { static constexpr int value = %d; };'
      % (cls + (BLOCKS_HINT.get(tuple(cls), 0),)))
    w('template <> struct StageBra<%d, %d, %d, %d> { static constexpr bool value = %s; };'
      % (cls + ('true' if tuple(cls) in STAGE_BRA else 'false',)))
    w('template <> struct AccumulateJ<%d, %d, %d, %d> { static constexpr int value = %d; };'
      % (cls + (ACCUM_J.get(tuple(cls), 0),)))
    w(g.emit(parts=class_parts(cls)))
    w('')
    w('void launch_quartet_%s(int mode, const FockArgs& a, int grid, cudaStream_t st)' % nm)
    w('{')
    w('    const dim3 blk(32 * kWarpsPerBlock);')
    w('    if (needs_ext(a))')
    w('        quartet_kernel_of<%d, %d, %d, %d, true>()<<<grid, blk, 0, st>>>(a, mode);' % cls)
    w('    else')
    w('        quartet_kernel_of<%d, %d, %d, %d, false>()<<<grid, blk, 0, st>>>(a, mode);' % cls)
    w('}')
    w('int occupancy_quartet_%s(int ext)' % nm)
    w('{')
    w('    int n = 0;')
    w('    if (ext)')
    w('        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, quartet_kernel_of<%d, %d, %d, %d, true>(), 32 * kWarpsPerBlock, 0);' % cls)
    w('    else')
    w('        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, quartet_kernel_of<%d, %d, %d, %d, false>(), 32 * kWarpsPerBlock, 0);' % cls)
    w('    return n;')
    w('}')
    if (la, lb) == (lc, ld):
        w('void launch_schwarz_%d%d(const PairBlockDev* blocks, int bid, int npairs, const double* boys, double* maxv, cudaStream_t st)' % (la, lb))
        w('{')
        w('    if (npairs > 0) schwarz_kernel<%d, %d><<<(npairs + 63) / 64, 64, 0, st>>>(blocks, bid, boys, maxv);' % (la, lb))
        w('}')
    w('}  // namespace vlx')
    text = '\n'.join(body) + '\n'
    path = outdir / ('class_%s.cu' % nm)
    if not path.exists() or path.read_text() != text:
        path.write_text(text)
    return path, g.stats()


VRR_COMPILED_MAX = 2400
ACC_COMPILED_MAX = 180


# Classes beyond the register budget that are compiled all the same (the
# compiler keeps what does not fit the registers in thread-local memory),
# with the number of accumulator groups of ClassGen.emit: measured faster
# than the warp-cooperative kernel on the (H2O)64 / def2-TZVP build.  The
# group counts are the fastest of a sweep over about 1.5x, 2x and 3x the
# earlier counts on that build (more groups: a smaller live set per group,
# fewer spills, at the cost of re-running the recursion per group); the
# sweep took the grouped classes from 1.33 s to 0.90 s of the build.
GROUPED = {(1, 2, 1, 2): 5, (1, 3, 0, 3): 5, (1, 3, 1, 1): 5, (1, 3, 1, 2): 6, (1, 3, 1, 3): 10, (1, 3, 2, 2): 12,
           (2, 2, 0, 2): 3, (2, 2, 0, 3): 5, (2, 2, 1, 1): 3, (2, 2, 1, 2): 8, (2, 2, 2, 2): 16, (2, 3, 0, 2): 5,
           (2, 3, 0, 3): 12, (2, 3, 1, 1): 6, (2, 3, 1, 2): 15, (2, 3, 1, 3): 16, (3, 3, 0, 1): 3, (3, 3, 0, 2): 9,
           (3, 3, 0, 3): 15, (3, 3, 1, 1): 10, (3, 3, 1, 2): 16}


# Minimum resident 128-thread blocks per SM a class's register allocation
# must allow (absent: no minimum).  4 for classes whose unconstrained
# allocation (164-168 registers, 3 blocks) fits 128 registers without
# spilling (measured 15-20% faster each); a minimum of 3 for the classes at
# 250+ registers was measured neutral.  An explicit minimum of 1 is not the
# same as none: it lets the compiler take far more registers (186 instead of
# 72 for (sp|ss)).  After the Fock additions became reductions without a
# returned value, (pp|ss) 6, (sd|ss) 8 and (sp|sp) 6 measured 1-13% faster
# than 4, 5 and 5; higher minimums for (sp|ss), (pp|sp) and (sd|sp) were
# slower (up to 1.8x).
BLOCKS_HINT = {(1, 1, 0, 0): 6, (0, 1, 0, 1): 6, (0, 2, 0, 0): 8, (0, 1, 0, 0): 8, (1, 1, 0, 1): 4, (0, 2, 0, 1): 4}

# Classes whose bra primitive records are staged in shared memory per work
# item: measured faster staged on the (H2O)32 / def2-SVP build ((ss|ss)
# 1.19x, (sp|ss) 1.08x, (pp|ss) 1.05x, (sd|ss) 1.03x, (dd|pd) 1.46x); the
# other classes measured neutral to slower (down to 0.34x for (dd|dd)).
STAGE_BRA = {(0, 0, 0, 0), (0, 1, 0, 0), (1, 1, 0, 0), (0, 2, 0, 0), (2, 2, 1, 2)}


# Classes whose plain kernels sum the J elements of the bra block F_PQ per
# work item (1: in registers, 2: in a per-warp shared-memory array) instead of
# one warp sum and atomic add per 32-ket step (absent: per step).  Chosen per
# class from timings of all three forms on the (H2O)32 / def2-SVP and
# (H2O)64 / def2-TZVP builds (gains 3-12% per class; (sp|ss), (sp|sp),
# (ss|ss), (pd|pd), (pd|pp), (sf|sf), (sf|pp) measured neutral or slower and
# stay per step).
ACCUM_J = {(1, 1, 0, 1): 1, (1, 2, 0, 1): 2, (1, 1, 0, 0): 2, (0, 2, 0, 1): 2, (0, 2, 1, 1): 2, (0, 2, 0, 0): 2,
           (1, 1, 1, 1): 2, (1, 2, 0, 2): 2, (1, 2, 0, 0): 1, (0, 3, 0, 1): 2, (0, 3, 1, 2): 1, (0, 3, 0, 0): 2,
           (0, 3, 0, 2): 2}


def class_parts(cls):
    return GROUPED.get(tuple(cls), 1)


def is_compiled(cls):
    """Straight-line per-lane kernel when the contracted buffer and the
    recursion graph are small enough, or the class is listed in GROUPED;
    otherwise the warp-cooperative kernel."""
    if tuple(cls) in GROUPED:
        return True
    g = ClassGen(*cls)
    return len(g.vrr.order) <= VRR_COMPILED_MAX and len(g.e_targets) * len(g.f_targets) <= ACC_COMPILED_MAX


def emit_dispatch(compiled, lmax, outdir):
    lines = ['// Generated by gen_eri.py -- do not edit.', '#pragma once', 'namespace vlx {']
    for c in compiled:
        nm = class_name(c)
        lines.append('void launch_quartet_%s(int mode, const FockArgs& a, int grid, cudaStream_t st);' % nm)
        lines.append('int occupancy_quartet_%s(int mode);' % nm)
    schw = [(a, b) for (a, b) in pair_classes(lmax) if (a, b, a, b) in compiled]
    for (a, b) in schw:
        lines.append('void launch_schwarz_%d%d(const PairBlockDev* blocks, int bid, int npairs, const double* boys, double* maxv, cudaStream_t st);' % (a, b))
    lines.append('struct QuartetClassEntry { int la, lb, lc, ld; void (*launch)(int, const FockArgs&, int, cudaStream_t); int (*occupancy)(int); int prim_flops, post_flops; };')
    lines.append('static const QuartetClassEntry kQuartetClasses[] = {')
    for c in compiled:
        nm = class_name(c)
        fv, fa, fp = ClassGen(*c).flops()
        lines.append('    {%d, %d, %d, %d, launch_quartet_%s, occupancy_quartet_%s, %d, %d},' % (c + (nm, nm, fv + fa, fp)))
    lines.append('};')
    lines.append('static const int kNumQuartetClasses = %d;' % len(compiled))
    lines.append('struct SchwarzEntry { int la, lb; void (*launch)(const PairBlockDev*, int, int, const double*, double*, cudaStream_t); };')
    lines.append('static const SchwarzEntry kSchwarzClasses[] = {')
    for (a, b) in schw:
        lines.append('    {%d, %d, launch_schwarz_%d%d},' % (a, b, a, b))
    lines.append('};')
    lines.append('static const int kNumSchwarzClasses = %d;' % len(schw))
    lines.append('}  // namespace vlx')
    text = '\n'.join(lines) + '\n'
    path = outdir / 'dispatch.inc'
    if not path.exists() or path.read_text() != text:
        path.write_text(text)


def emit_sph_table(outdir, lmax=4):
    """Spherical factors for l <= lmax as a constant table [l][m][cart]
    (m = 0..2l for -l..l, lexicographic Cartesian components)."""
    vals = []
    for l in range(lmax + 1):
        rows = sph_coefficients(l)
        for m in range(9):
            for c in range(15):
                vals.append(rows[m][c] if (m < 2 * l + 1 and c < ncart(l)) else 0.0)
    text = ('// Generated by gen_eri.py -- do not edit.\n#pragma once\n'
            '#define VLX_SPH_LMAX %d\n' % lmax +
            '__constant__ double c_sph[%d] = {%s};\n' % (len(vals), ', '.join(repr(v) for v in vals)))
    path = outdir / 'sph_table.inc'
    if not path.exists() or path.read_text() != text:
        path.write_text(text)


def _lin_expr(terms):
    """sum of (coefficient, name) terms as T-typed code ('T(0)' if empty)."""
    parts = ['T(%s) * %s' % (_num(c), n) for c, n in terms if c != 0.0]
    return ' + '.join(parts) if parts else 'T(0)'


def ket_xform_code(lc, ld):
    """Ket half of the post-contraction steps for one bra component e: ket
    HRR |c+1_i, d) = |c, d+1_i) + (D_i - C_i)|c, d) on the Cartesian f-vector
    [e 0 | f 0], f in [ld, lc+ld] (input in[jf], f_targets order), then the
    ket Cartesian -> spherical transform; output out[(k nd + l) os]."""
    f_t = [c for l in range(ld, lc + ld + 1) for c in cart_list(l)]
    f_index = {f: j for j, f in enumerate(f_t)}
    nodes, order = {}, []

    def need(c, d):
        key = (c, d)
        if key in nodes:
            return key
        if sum(c) == 0:
            nodes[key] = ('F', f_index[d])
        else:
            i = pick_axis(c)
            c1 = sub1(c, i)
            nodes[key] = ('H', i, need(c1, add1(d, i)), need(c1, d))
        order.append(key)
        return key

    cc, dc = cart_list(lc), cart_list(ld)
    for c in cc:
        for d in dc:
            need(c, d)
    names = {}
    body = []
    for n_, key in enumerate(order):
        node = nodes[key]
        nm = 'k%d' % n_
        names[key] = nm
        if node[0] == 'F':
            body.append('        const T %s = in[%d];' % (nm, node[1]))
        else:
            body.append('        const T %s = %s + DC%s * %s;' % (nm, names[node[2]], AX[node[1]], names[node[3]]))
    sc, sd = sph_coefficients(lc), sph_coefficients(ld)
    nc, nd = 2 * lc + 1, 2 * ld + 1
    for k in range(nc):
        for l in range(nd):
            terms = [(sc[k][ic] * sd[l][jd], names[(c, d)]) for ic, c in enumerate(cc) for jd, d in enumerate(dc)
                     if sc[k][ic] != 0.0 and sd[l][jd] != 0.0]
            body.append('        out[%d * os] = %s;' % (k * nd + l, _lin_expr(terms)))
    head = ['template <> struct KetXform<%d, %d> {' % (lc, ld),
            '    static constexpr int NIN = %d, NOUT = %d;' % (len(f_t), nc * nd),
            '    template <typename T>',
            '    __device__ __forceinline__ static void run(const T* __restrict__ in, T* __restrict__ out, const int os,',
            '                                               const T DCx, const T DCy, const T DCz)',
            '    {',
            '        (void)DCx; (void)DCy; (void)DCz;']
    return '\n'.join(head + body + ['    }', '};', ''])


def bra_xform_code(la, lb):
    """Bra half for one half-spherical ket component: bra HRR
    (a+1_i, b| = (a, b+1_i| + (B_i - A_i)(a, b| on the e-vector, e in
    [lb, la+lb] (input in[ie is], e_targets order), then the bra Cartesian ->
    spherical transform; output out[(i nb + j) os]."""
    e_t = [c for l in range(lb, la + lb + 1) for c in cart_list(l)]
    e_index = {e: j for j, e in enumerate(e_t)}
    nodes, order = {}, []

    def need(a, b):
        key = (a, b)
        if key in nodes:
            return key
        if sum(a) == 0:
            nodes[key] = ('E', e_index[b])
        else:
            i = pick_axis(a)
            a1 = sub1(a, i)
            nodes[key] = ('H', i, need(a1, add1(b, i)), need(a1, b))
        order.append(key)
        return key

    ac, bc = cart_list(la), cart_list(lb)
    for a in ac:
        for b in bc:
            need(a, b)
    names = {}
    body = []
    for n_, key in enumerate(order):
        node = nodes[key]
        nm = 'b%d' % n_
        names[key] = nm
        if node[0] == 'E':
            body.append('        const T %s = in[%d * is];' % (nm, node[1]))
        else:
            body.append('        const T %s = %s + BA%s * %s;' % (nm, names[node[2]], AX[node[1]], names[node[3]]))
    sa, sb = sph_coefficients(la), sph_coefficients(lb)
    na, nb = 2 * la + 1, 2 * lb + 1
    for i in range(na):
        for j in range(nb):
            terms = [(sa[i][ia] * sb[j][jb], names[(a, b)]) for ia, a in enumerate(ac) for jb, b in enumerate(bc)
                     if sa[i][ia] != 0.0 and sb[j][jb] != 0.0]
            body.append('        out[%d * os] = %s;' % (i * nb + j, _lin_expr(terms)))
    head = ['template <> struct BraXform<%d, %d> {' % (la, lb),
            '    static constexpr int NIN = %d, NOUT = %d;' % (len(e_t), na * nb),
            '    template <typename T>',
            '    __device__ __forceinline__ static void run(const T* __restrict__ in, const int is, T* __restrict__ out,',
            '                                               const int os, const T BAx, const T BAy, const T BAz)',
            '    {',
            '        (void)BAx; (void)BAy; (void)BAz;']
    return '\n'.join(head + body + ['    }', '};', ''])


def emit_xforms(outdir, lmax, interp):
    """xform.inc: the compiled ket / bra transforms of every pair class, and
    coop_classes.inc: one VLX_COOP_CLASS(la, lb, lc, ld) line per
    warp-cooperative class."""
    out = ['// generated by gen_eri.py: post-contraction transforms (HRR + Cartesian -> spherical)',
           'template <int LC, int LD> struct KetXform;', 'template <int LA, int LB> struct BraXform;', '']
    for a, b in pair_classes(lmax):
        out.append(ket_xform_code(a, b))
        out.append(bra_xform_code(a, b))
    text = '\n'.join(out)
    path = outdir / 'xform.inc'
    if not path.exists() or path.read_text() != text:
        path.write_text(text)
    lines = ['// generated by gen_eri.py: warp-cooperative quartet classes'] + \
            ['VLX_COOP_CLASS(%d, %d, %d, %d)' % c for c in interp]
    text = '\n'.join(lines) + '\n'
    path = outdir / 'coop_classes.inc'
    if not path.exists() or path.read_text() != text:
        path.write_text(text)


def main():
    outdir = Path(sys.argv[1])
    lmax = int(sys.argv[2]) if len(sys.argv) > 2 else 3
    outdir.mkdir(parents=True, exist_ok=True)
    classes = quartet_classes(lmax)
    compiled = [c for c in classes if is_compiled(c)]
    interp = [c for c in classes if not is_compiled(c)]
    for p in ('interp_programs.bin',):
        if (outdir / p).exists():
            (outdir / p).unlink()
    for cls in compiled:
        emit_class_file(cls, outdir)
    emit_dispatch(compiled, lmax, outdir)
    emit_sph_table(outdir)
    emit_xforms(outdir, lmax, interp)
    import gen_coop
    gen_coop.emit_blob(interp, outdir / 'coop_programs.bin')
    for p in outdir.glob('class_*.cu'):
        if tuple(int(ch) for ch in p.stem[6:]) not in compiled:
            p.unlink()
    print('compiled classes:', len(compiled), 'warp-cooperative classes:', len(interp))


if __name__ == '__main__':
    main()
