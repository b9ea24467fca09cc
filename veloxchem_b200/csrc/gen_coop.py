"""Warp-cooperative recursion programs for the large quartet classes.

For classes whose contracted buffer does not fit in registers, one warp
evaluates one shell quartet: the recursion graph of gen_eri.ClassGen (the same
Obara-Saika VRR on B and D, contraction, ket HRR, ket Cartesian->spherical,
bra HRR, bra Cartesian->spherical) is turned into a list of operations on a
per-warp shared-memory array, ASAP-scheduled into levels (every operation of a
level is independent, lanes take them round-robin, __syncwarp between levels)
and slot-allocated by liveness, so that a slot freed at level u is reused from
level u + 1 on.

Operations (executed by vlx_coop.cu):
  VRR  kind 0 (bra, G = P-B, W-P) / 1 (ket, G = Q-D, W-Q), axis a:
       S[t] = G1[a] S[x] + G2[a] S[y] + c1 H (S[u] - R S[v]) + c2 hizh S[w]
  ACC  kind 2: S[t] += S[x]   (contracted accumulator, once per primitive quartet)
  HRR  kind 3 (ket, D - C) / 4 (bra, B - A), axis a: S[t] = S[x] + G[a] S[y]
  LIN  kind 5: S[t] = w0 S[x] + w1 S[y] + w2 S[u]   (one index of a spherical transform)
Slot 0 holds 0.0; slots 1..nacc hold the contracted accumulators; the Boys
values pref * F_m are written to their slots before the VRR levels.
"""

import struct

from gen_eri import ClassGen, add1, cart_list, pick_axis, sph_coefficients, sub1


class Op:
    __slots__ = ('kind', 'axis', 'dst', 'src', 'c1', 'c2', 'w', 'level')

    def __init__(self, kind, axis, dst, src, c1=0, c2=0, w=None):
        self.kind, self.axis, self.dst, self.src = kind, axis, dst, src
        self.c1, self.c2, self.w = c1, c2, w or (0.0, 0.0, 0.0)
        self.level = 0


class CoopProgram:
    def __init__(self, la, lb, lc, ld):
        self.cls = (la, lb, lc, ld)
        g = ClassGen(la, lb, lc, ld)
        self.g = g
        self.L = g.L
        nid = [0]

        def new():
            nid[0] += 1
            return nid[0]

        ZERO = 0
        val = {}          # VRR key -> value id
        self.fvals = {}   # m -> value id
        body = []
        for key in g.vrr.order:
            terms = g.vrr.nodes[key]
            if terms[0][0] == 'BASE':
                m = terms[0][1]
                if m not in self.fvals:
                    self.fvals[m] = new()
                val[key] = self.fvals[m]
                continue
            kind = 1 if terms[0][0] in ('QD', 'WQ') else 0
            axis = terms[0][1]
            x, y = val[terms[0][2]], val[terms[1][2]]
            u = v = w = ZERO
            c1 = c2 = 0
            for t in terms[2:]:
                if t[0] in ('F2', 'E2'):
                    c1 = t[1]
                    u, v = val[t[2]], val[t[3]]
                elif t[0] == 'EZH':
                    c2 = t[1]
                    w = val[t[2]]
            d = new()
            val[key] = d
            body.append(Op(kind, axis, d, [x, y, u, v, w], c1, c2))
        # accumulators: fixed slots 1..nacc
        self.acc = {}
        acc_ops = []
        for e in g.e_targets:
            for f in g.f_targets:
                a = new()
                self.acc[(e, f)] = a
                acc_ops.append(Op(2, 0, a, [val[(e, f, 0)]]))
        self.body = body
        self.acc_ops = acc_ops
        # post: ket HRR, ket sph (c then d), bra HRR, bra sph (a then b)
        post = []
        cc, dc = cart_list(lc), cart_list(ld)
        ac, bc = cart_list(la), cart_list(lb)
        sc, sd = sph_coefficients(lc), sph_coefficients(ld)
        sa, sb = sph_coefficients(la), sph_coefficients(lb)
        nc_, nd_, na_, nb_ = 2 * lc + 1, 2 * ld + 1, 2 * la + 1, 2 * lb + 1

        def lin(terms):
            """value = sum w_k v_k, split into LIN ops of up to 3 terms."""
            terms = [(w_, v_) for (w_, v_) in terms if w_ != 0.0]
            acc_v = None
            while terms:
                chunk = terms[:3] if acc_v is None else [(1.0, acc_v)] + terms[:2]
                terms = terms[3:] if acc_v is None else terms[2:]
                while len(chunk) < 3:
                    chunk.append((0.0, ZERO))
                d = new()
                post.append(Op(5, 0, d, [chunk[0][1], chunk[1][1], chunk[2][1]], w=tuple(c[0] for c in chunk)))
                acc_v = d
            return acc_v if acc_v is not None else ZERO

        h = {}
        for e in g.e_targets:
            kn = {}

            def need_ket(c, dd):
                if (c, dd) in kn:
                    return kn[(c, dd)]
                if sum(c) == 0:
                    kn[(c, dd)] = self.acc[(e, dd)]
                else:
                    i = pick_axis(c)
                    c1_ = sub1(c, i)
                    x = need_ket(c1_, add1(dd, i))
                    y = need_ket(c1_, dd)
                    t = new()
                    post.append(Op(3, i, t, [x, y]))
                    kn[(c, dd)] = t
                return kn[(c, dd)]

            for c in cc:
                for dd in dc:
                    need_ket(c, dd)
            # transform c, then d
            half = {}
            for k in range(nc_):
                for jd, dd in enumerate(dc):
                    half[(k, jd)] = lin([(sc[k][ic], kn[(c, dd)]) for ic, c in enumerate(cc)])
            for k in range(nc_):
                for l in range(nd_):
                    h[(e, k, l)] = lin([(sd[l][jd], half[(k, jd)]) for jd in range(len(dc))])
        self.out = [0] * (na_ * nb_ * nc_ * nd_)
        for k in range(nc_):
            for l in range(nd_):
                bn = {}

                def need_bra(a, b):
                    if (a, b) in bn:
                        return bn[(a, b)]
                    if sum(a) == 0:
                        bn[(a, b)] = h[(b, k, l)]
                    else:
                        i = pick_axis(a)
                        a1 = sub1(a, i)
                        x = need_bra(a1, add1(b, i))
                        y = need_bra(a1, b)
                        t = new()
                        post.append(Op(4, i, t, [x, y]))
                        bn[(a, b)] = t
                    return bn[(a, b)]

                for a in ac:
                    for b in bc:
                        need_bra(a, b)
                halfb = {}
                for i in range(na_):
                    for jb, b in enumerate(bc):
                        halfb[(i, jb)] = lin([(sa[i][ia], bn[(a, b)]) for ia, a in enumerate(ac)])
                for i in range(na_):
                    for j in range(nb_):
                        self.out[((i * nb_ + j) * nc_ + k) * nd_ + l] = \
                            lin([(sb[j][jb], halfb[(i, jb)]) for jb in range(len(bc))])
        self.post = post
        self._schedule()

    # ------------------------------------------------------------ scheduling
    def _schedule(self):
        # body: F values at level 0, ASAP levels, ACC right after its source
        lvl = {0: 0}
        for m, v in self.fvals.items():
            lvl[v] = 0
        for op in self.body:
            op.level = 1 + max(lvl[s] for s in op.src)
            lvl[op.dst] = op.level
        for op in self.acc_ops:
            op.level = lvl[op.src[0]] + 1
        self.body_levels = max([op.level for op in self.body + self.acc_ops] + [0])
        # post: accumulators at level 0
        plvl = {0: 0}
        for a in self.acc.values():
            plvl[a] = 0
        for op in self.post:
            op.level = 1 + max(plvl[s] for s in op.src)
            plvl[op.dst] = op.level
        self.post_levels = max([op.level for op in self.post] + [0])
        self._allocate()

    def _allocate(self):
        """Slot allocation: 0 = zero, 1..nacc = accumulators, then a shared pool
        for body values (live within one primitive iteration) and post values."""
        nacc = len(self.acc)
        slot = {0: 0}
        for n, a in enumerate(sorted(self.acc.values())):
            slot[a] = 1 + n
        base = 1 + nacc

        def alloc(defs_by_level, last_use, nlev, preset):
            # defs_by_level[l] = values defined at level l; last_use[v] = level
            free, top = [], [base]
            release = {}
            for v, u in last_use.items():
                release.setdefault(u, []).append(v)
            for l in range(nlev + 1):
                for v in defs_by_level.get(l, []):
                    if v in preset:
                        continue
                    if free:
                        slot[v] = free.pop()
                    else:
                        slot[v] = top[0]
                        top[0] += 1
                # slots of values whose last use is level l become free after level l
                for v in release.get(l, []):
                    if v in slot and v not in preset and slot[v] >= base:
                        free.append(slot[v])
            return top[0]

        # body
        defs, last = {}, {}
        for m, v in self.fvals.items():
            defs.setdefault(0, []).append(v)
            last[v] = 0
        for op in self.body:
            defs.setdefault(op.level, []).append(op.dst)
            last.setdefault(op.dst, op.level)
        for op in self.body + self.acc_ops:
            for s in op.src:
                if s != 0 and s not in self.acc.values():
                    last[s] = max(last.get(s, 0), op.level)
        preset = set(self.acc.values()) | {0}
        top_body = alloc(defs, last, self.body_levels, preset)
        # post (body values are dead): accumulators released after their last use
        defs, last = {}, {}
        outs = set(self.out)
        for op in self.post:
            defs.setdefault(op.level, []).append(op.dst)
            last.setdefault(op.dst, op.level)
        for op in self.post:
            for s in op.src:
                if s != 0:
                    last[s] = max(last.get(s, 0), op.level)
        for v in outs:
            last[v] = self.post_levels + 1
        # accumulator slots become reusable after their last use in post
        acc_set = set(self.acc.values())
        top_post = self._alloc_post(defs, last, acc_set, slot, base)
        self.slot = slot
        self.nslots = max(top_body, top_post)

    def _alloc_post(self, defs, last, acc_set, slot, base):
        free, top = [], base
        release = {}
        for v, u in last.items():
            release.setdefault(u, []).append(v)
        for v in acc_set:
            if v not in last:
                release.setdefault(0, []).append(v)
        for l in range(self.post_levels + 2):
            for v in defs.get(l, []):
                if free:
                    slot[v] = free.pop()
                else:
                    slot[v] = top
                    top += 1
            for v in release.get(l, []):
                if v in slot and v != 0:
                    free.append(slot[v])
        return top

    # ------------------------------------------------------------ emission
    def records(self):
        """(level-sorted ops, level offsets) for body, acc merged into body levels, and post."""
        s = self.slot
        # inside a level, group operations of one kind so that a warp's
        # 32-wide round executes one code path
        body = sorted(self.body + self.acc_ops, key=lambda o: (o.level, o.kind))
        post = sorted(self.post, key=lambda o: (o.level, o.kind))

        def offsets(ops, nlev):
            off = [0] * (nlev + 2)
            for o in ops:
                off[o.level + 1] += 1
            for l in range(1, nlev + 2):
                off[l] += off[l - 1]
            return off

        return body, offsets(body, self.body_levels), post, offsets(post, self.post_levels)

    def pack(self):
        """16-byte op records: int32 {dst | x << 16, y | u << 16, v | w << 16,
        kind*4+axis | c1 << 8 | c2 << 16}; a LIN op keeps its 3 weights in the
        class's weight array and their index in the (v | w << 16) word."""
        s = self.slot
        body, boff, post, poff = self.records()
        ints, lw = [], []
        for o in body + post:
            src = [s[x] for x in o.src] + [0] * (5 - len(o.src))
            assert max(src + [s[o.dst]]) < 65536
            if o.kind == 5:
                word2 = len(lw) // 3
                lw.extend(o.w)
            else:
                word2 = src[3] | (src[4] << 16)
            ints.append(struct.pack('<4i', s[o.dst] | (src[0] << 16), src[1] | (src[2] << 16), word2,
                                    (o.kind * 4 + o.axis) | ((o.c1 & 0xff) << 8) | ((o.c2 & 0xff) << 16)))
        fslots = [s[self.fvals[m]] if m in self.fvals else 0 for m in range(self.L + 1)]
        outs = [s[v] for v in self.out]
        return dict(ints=b''.join(ints), lw=lw, nbody=len(body), npost=len(post),
                    boff=boff, poff=poff, fslots=fslots, outs=outs, nslots=self.nslots, nacc=len(self.acc))


def emit_blob(classes, path):
    """Binary blob of the cooperative programs (embedded by vlx_blob.S).

    int32 magic 0x434F4F51, int32 count; per class 16 int32 header
    (la lb lc ld nslots nacc nbody npost nbody_levels npost_levels op_offset
    aux_offset prim_flops post_flops weight_offset nweights); then all op
    records (4 int32 each); then all LIN weights (float64); then the aux int32
    stream per class: body level offsets (nbody_levels + 2), post level offsets
    rebased after the body ops (npost_levels + 2), F slots (L + 1), output slots."""
    heads, ops, wts, aux = [], [], [], []
    nops = naux = nw = 0
    for cls in classes:
        p = CoopProgram(*cls)
        r = p.pack()
        a = r['boff'] + [x + r['nbody'] for x in r['poff']] + r['fslots'] + r['outs']
        fv, fa, fp = p.g.flops()
        heads.append(struct.pack('<16i', *cls, r['nslots'], r['nacc'], r['nbody'], r['npost'], len(r['boff']) - 2,
                                 len(r['poff']) - 2, nops, naux, fv + fa, fp, nw, len(r['lw'])))
        ops.append(r['ints'])
        wts.append(struct.pack('<%dd' % len(r['lw']), *r['lw']))
        aux.append(struct.pack('<%di' % len(a), *a))
        nops += r['nbody'] + r['npost']
        naux += len(a)
        nw += len(r['lw'])
    blob = (struct.pack('<2i', 0x434F4F51, len(classes)) + b''.join(heads) + b''.join(ops) + b''.join(wts) +
            b''.join(aux))
    if not path.exists() or path.read_bytes() != blob:
        path.write_bytes(blob)


if __name__ == '__main__':
    import sys
    for cls in [(1, 2, 1, 2), (2, 2, 1, 1), (2, 2, 0, 2), (2, 2, 1, 2), (2, 2, 2, 2), (3, 3, 3, 3)]:
        p = CoopProgram(*cls)
        nb = len(p.body) + len(p.acc_ops)
        print(cls, 'slots', p.nslots, 'acc', len(p.acc), 'body ops', nb, 'levels', p.body_levels,
              'post ops', len(p.post), 'levels', p.post_levels, 'smem/warp KB %.1f' % (p.nslots * 8 / 1024))
        sys.stdout.flush()
