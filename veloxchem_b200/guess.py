"""Learned initial density guess for water clusters (def2-SVP).

The reference starts its SCF from SAD (src/pymodule/sadguessdriver.py); this
module adds a guess predicted by a small network, with SAD as the fallback.

Representation.  The alpha density D (D = C_occ C_occ^T, the matrix the SCF
driver iterates) is cut into atom-pair blocks D_ij (rows: the AOs of atom i,
columns: those of atom j).  Each block is expressed in local frames: every
atom takes the frame of its water molecule (origin O, e1 along the HOH
bisector, e3 normal to the molecular plane, e2 = e3 x e1), and

    B_ij = R_i^T D_ij R_j

where R_i is the block-diagonal rotation of the real solid harmonics of atom
i's shells for that frame.  B_ij is invariant under rigid rotations and
translations of the cluster, and so is the pair descriptor: element pair,
distance, the pair vector and relative orientation in the two frames, the
atoms' positions in their waters, and radial neighbour densities and the
first and second moments of the neighbour directions within 5 Angstrom.  The network predicts B_ij - B_ij(SAD) for all
pairs closer than PAIR_CUTOFF; blocks beyond it are zero.  The assembled
matrix is symmetrised and replaced by the nearest idempotent density with
N_occ electrons (its N_occ natural orbitals of largest occupation).

Fallback rule: the SCF driver evaluates the energy of the first iteration
from both the learned and the SAD density and keeps the lower one.
"""

import math
from pathlib import Path

import numpy as np

BOHR_IN_ANGSTROM = 0.529177210903
PAIR_CUTOFF = 5.0       # Angstrom
ENV_CUTOFF = 5.0        # Angstrom
RBF_CENTERS = np.linspace(1.0, 5.0, 8)
RBF_WIDTH = 0.5
MOM_CENTERS = np.array([1.5, 2.5, 3.5, 4.5])
MOM_WIDTH = 0.7
NTYPES = 5              # self-O, self-H, O-O, O-H, H-H
NOUT = 196              # largest block: O x O in def2-SVP (14 x 14)
NENV = 2 * len(RBF_CENTERS) + 3 * len(MOM_CENTERS) + 6 * len(MOM_CENTERS)  # per atom
NFEAT = NTYPES + 1 + 3 + 3 + 3 + 9 + 3 + 3 + 2 * NENV

WEIGHTS = Path(__file__).resolve().parent / 'data' / 'guess_mlp_svp.npz'


# ------------------------------------------------------------ real solid harmonics

def _solid_harmonics(l, r):
    """Real solid harmonics of the reference's AO convention (m = -l..l;
    src/general/SphericalMomentum.hpp: p as (y, z, x); d as 2 sqrt3 xy,
    2 sqrt3 yz, 2z^2 - x^2 - y^2, 2 sqrt3 xz, sqrt3 (x^2 - y^2))."""
    x, y, z = r[:, 0], r[:, 1], r[:, 2]
    if l == 0:
        return np.ones((len(r), 1))
    if l == 1:
        return np.stack([y, z, x], axis=1)
    if l == 2:
        f3 = 2.0 * math.sqrt(3.0)
        return np.stack([f3 * x * y, f3 * y * z, 2 * z * z - x * x - y * y, f3 * x * z,
                         0.5 * f3 * (x * x - y * y)], axis=1)
    raise ValueError('learned guess: l > 2 not needed for def2-SVP water')


_SAMPLE = np.random.default_rng(12345).standard_normal((64, 3))


def sh_rotation(l, Q):
    """Matrix D with Y_m(Q^T r) = sum_m' D[m', m] Y_m'(r): the AO coefficients
    of a shell transform as c' = D c when the molecule is rotated by Q."""
    a = _solid_harmonics(l, _SAMPLE)
    b = _solid_harmonics(l, _SAMPLE @ Q)  # rows: (Q^T r)^T = r^T Q
    d, *_ = np.linalg.lstsq(a, b, rcond=None)
    return d


def atom_rotation(shell_ls, Q):
    """Block-diagonal AO rotation of one atom's shells (in atom AO order)."""
    mats = [sh_rotation(l, Q) for l in shell_ls]
    n = sum(m.shape[0] for m in mats)
    out = np.zeros((n, n))
    o = 0
    for m in mats:
        k = m.shape[0]
        out[o:o + k, o:o + k] = m
        o += k
    return out


# ------------------------------------------------------------ structure of a cluster

class ClusterLayout:
    """Atoms, AO lists, water frames and the pair list of one water cluster
    (all per-pair work vectorised over the pairs of one element pair)."""

    def __init__(self, molecule, basis):
        self.z = np.asarray(molecule.get_element_ids(), dtype=np.int64)
        self.xyz = np.asarray(molecule.get_coordinates_in_bohr(), dtype=np.float64) * BOHR_IN_ANGSTROM
        n = len(self.z)
        aos = basis.ao_indices()
        self.atom_aos = [[] for _ in range(n)]
        self.atom_ls = [[] for _ in range(n)]
        for s, idx in zip(basis.shells, aos):
            self.atom_aos[s.atom].extend(int(i) for i in idx)
            self.atom_ls[s.atom].append(s.l)
        self.atom_aos = [np.array(a, dtype=np.int64) for a in self.atom_aos]
        self.nao = basis.get_dimensions_of_basis()
        self._frames()
        self._pairs()

    def _frames(self):
        z, xyz = self.z, self.xyz
        oxy = np.where(z == 8)[0]
        hyd = np.where(z == 1)[0]
        if len(oxy) == 0 or len(hyd) != 2 * len(oxy) or len(z) != 3 * len(oxy):
            raise ValueError('learned guess: molecule is not a water cluster')
        owner = np.argmin(np.linalg.norm(xyz[hyd][:, None, :] - xyz[oxy][None, :, :], axis=2), axis=1)
        self.water = np.zeros(len(z), dtype=np.int64)
        self.water[oxy] = np.arange(len(oxy))
        self.water[hyd] = owner
        self.frames = np.zeros((len(oxy), 3, 3))
        self.origin = xyz[oxy]
        for w, o in enumerate(oxy):
            hs = hyd[owner == w]
            if len(hs) != 2:
                raise ValueError('learned guess: oxygen without exactly two hydrogens')
            u1, u2 = xyz[hs[0]] - xyz[o], xyz[hs[1]] - xyz[o]
            e1 = u1 + u2
            e1 /= np.linalg.norm(e1)
            e3 = np.cross(u1, u2)
            e3 /= np.linalg.norm(e3)
            e2 = np.cross(e3, e1)
            self.frames[w] = np.stack([e1, e2, e3], axis=1)  # columns: local axes in global coordinates
        # shell rotations per water (the frame rotation is Q = F^T), assembled per atom
        per_water = [{l: sh_rotation(l, self.frames[w].T) for l in (0, 1, 2)} for w in range(len(oxy))]
        self.rot = []
        for a in range(len(z)):
            mats = [per_water[self.water[a]][l] for l in self.atom_ls[a]]
            k = sum(m.shape[0] for m in mats)
            r = np.zeros((k, k))
            o = 0
            for m in mats:
                r[o:o + m.shape[0], o:o + m.shape[0]] = m
                o += m.shape[0]
            self.rot.append(r)

    def _pairs(self):
        z, xyz = self.z, self.xyz
        n = len(z)
        dist = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2)
        self.dist = dist
        ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing='ij')
        keep = (ii != jj) & (dist <= PAIR_CUTOFF)
        keep &= ~((z[:, None] == z[None, :]) & (jj < ii))
        keep &= ~((z[:, None] == 1) & (z[None, :] == 8))
        i2, j2 = np.nonzero(keep)
        self.pairs = np.concatenate([np.stack([np.arange(n), np.arange(n)], axis=1),
                                     np.stack([i2, j2], axis=1)]).astype(np.int64)
        # pairs grouped by element pair: the blocks of one group have one shape
        self.groups = []
        for zi, zj in ((8, 8), (8, 1), (1, 1)):
            sel = np.where((z[self.pairs[:, 0]] == zi) & (z[self.pairs[:, 1]] == zj))[0]
            if len(sel) == 0:
                continue
            a, b = self.pairs[sel, 0], self.pairs[sel, 1]
            self.groups.append((sel, np.stack([self.atom_aos[x] for x in a]), np.stack([self.atom_aos[x] for x in b]),
                                np.stack([self.rot[x] for x in a]), np.stack([self.rot[x] for x in b]),
                                a == b))

    # ---- descriptors
    def _env_all(self):
        """Radial O / H neighbour densities and the first and second moments
        (local frame; xx, yy, zz, xy, xz, yz) of the neighbour directions of
        every atom."""
        d = self.dist
        mask = (d > 1e-8) & (d < ENV_CUTOFF)
        out = []
        for el in (8, 1):
            w = (mask & (self.z[None, :] == el)).astype(np.float64)
            g = np.exp(-((d[:, :, None] - RBF_CENTERS[None, None, :]) / RBF_WIDTH) ** 2)
            out.append((g * w[:, :, None]).sum(axis=1))
        dsafe = np.where(mask, d, 1.0)
        v = (self.xyz[None, :, :] - self.xyz[:, None, :]) / dsafe[:, :, None]        # [i, n, 3]
        v = np.einsum('ink,ikl->inl', v, self.frames[self.water])                    # local frame of i
        g = np.exp(-((d[:, :, None] - MOM_CENTERS[None, None, :]) / MOM_WIDTH) ** 2) * mask[:, :, None]
        out.append(np.einsum('inc,inl->icl', g, v).reshape(len(self.z), -1))
        q = np.einsum('inc,inl,inm->iclm', g, v, v)
        iu = ([0, 1, 2, 0, 0, 1], [0, 1, 2, 1, 2, 2])
        out.append(q[:, :, iu[0], iu[1]].reshape(len(self.z), -1))
        return np.concatenate(out, axis=1)

    def descriptors(self):
        env = self._env_all()
        i, j = self.pairs[:, 0], self.pairs[:, 1]
        zi, zj = self.z[i], self.z[j]
        t = np.where(i == j, np.where(zi == 8, 0, 1), np.where((zi == 8) & (zj == 8), 2, np.where(zi == 8, 3, 4)))
        wa, wb = self.water[i], self.water[j]
        Fa, Fb = self.frames[wa], self.frames[wb]
        dv = self.xyz[j] - self.xyz[i]
        d = self.dist[i, j]
        cols = [np.eye(NTYPES)[t], (wa == wb)[:, None].astype(np.float64),
                np.stack([d, np.exp(-d), 1.0 / (1.0 + d)], axis=1),
                np.einsum('pk,pkl->pl', dv, Fa), np.einsum('pk,pkl->pl', dv, Fb),
                np.einsum('pkl,pkm->plm', Fa, Fb).reshape(len(i), 9),
                np.einsum('pk,pkl->pl', self.xyz[i] - self.origin[wa], Fa),
                np.einsum('pk,pkl->pl', self.xyz[j] - self.origin[wb], Fb), env[i], env[j]]
        return np.concatenate(cols, axis=1).astype(np.float32)

    # ---- blocks
    def local_blocks(self, D):
        """Local-frame blocks of D (row-major, padded to NOUT) and their mask."""
        T = np.zeros((len(self.pairs), NOUT), dtype=np.float32)
        M = np.zeros((len(self.pairs), NOUT), dtype=np.float32)
        for sel, ai, aj, ri, rj, _ in self.groups:
            blk = D[ai[:, :, None], aj[:, None, :]]
            b = ri @ blk @ np.swapaxes(rj, 1, 2)
            k = b.shape[1] * b.shape[2]
            T[sel, :k] = b.reshape(len(sel), k)
            M[sel, :k] = 1.0
        return T, M

    def assemble(self, B):
        """Global density from local-frame pair blocks (row-major, padded)."""
        D = np.zeros((self.nao, self.nao))
        for sel, ai, aj, ri, rj, same in self.groups:
            ni, nj = ai.shape[1], aj.shape[1]
            b = np.asarray(B[sel, :ni * nj], dtype=np.float64).reshape(len(sel), ni, nj)
            blk = np.swapaxes(ri, 1, 2) @ b @ rj
            off = ~same
            D[ai[off][:, None, :].transpose(0, 2, 1), aj[off][:, None, :]] = blk[off]
            D[aj[off][:, :, None], ai[off][:, None, :]] = np.swapaxes(blk[off], 1, 2)
            D[ai[same][:, :, None], aj[same][:, None, :]] = blk[same]
        return 0.5 * (D + D.T)


# ------------------------------------------------------------ the guess driver

_DRIVERS = {}


def learned_guess_driver(weights=None, device=0):
    """The driver of a weights file on a device, loaded once per process."""
    key = (str(WEIGHTS if weights is None else weights), int(device))
    if key not in _DRIVERS:
        _DRIVERS[key] = LearnedGuessDriver(weights, device)
    return _DRIVERS[key]


class LearnedGuessDriver:
    """Predicts the alpha density of a water cluster in def2-SVP from the
    trained network (BF16 inference on the GPU) on top of SAD."""

    def __init__(self, weights=None, device=0):
        from .guess_net import GuessMLP
        data = np.load(str(WEIGHTS if weights is None else weights))
        self.mu = data['mu'].astype(np.float32)
        self.sd = data['sd'].astype(np.float32)
        self.scale = float(data['target_scale'])
        depth = sum(1 for k in data.files if k.startswith('W'))
        width = data['W0'].shape[0]
        self.net = GuessMLP(data['W0'].shape[1], data['W%d' % (depth - 1)].shape[0], width, depth, device=device)
        self.net.load_state_dict(data)
        self.device = device

    def predict_any(self, molecule, basis, overlap, nocc, sad_density=None, ortho=None, refine_grad=None):
        """Learned alpha density in `basis`: predicted in def2-SVP and, for any
        other basis, carried over by the standard basis projection
        D = S_bb^-1 S_bs D_svp S_sb S_bb^-1 (b: target basis, s: def2-SVP)
        before the idempotent projection.  With refine_grad, the prediction is
        first refined by a loose def2-SVP SCF (gradient below refine_grad);
        measured on (H2O)64 / def2-TZVP this improved the first-iteration
        energy only from 3.0 to 2.7 Eh above the converged one for 3.6 s, so
        it is off by default."""
        import torch
        from . import _native as nat
        from .molecularbasis import MolecularBasis
        from .scf import SadGuessDriver
        if basis.name.upper() == 'DEF2-SVP' and sad_density is not None:
            return self.predict(molecule, basis, sad_density, overlap, nocc, ortho)
        svp = MolecularBasis.read(molecule, 'def2-svp')
        minb = MolecularBasis.read(molecule, 'ao-start-guess')
        s_svp = nat.one_electron(0, molecule, svp, None, self.device)
        d_sad = SadGuessDriver().compute(molecule, minb, svp, self.device, overlap=s_svp)
        d_svp = self.predict(molecule, svp, d_sad, s_svp, nocc)
        if basis.name.upper() == 'DEF2-SVP':
            return d_svp
        if refine_grad:
            from .scf import ScfRestrictedDriver
            drv = ScfRestrictedDriver(self.device)
            drv.conv_thresh = refine_grad
            drv.fp32_cutoff = 1.0e-5
            res = drv.compute(molecule, svp, guess_density=d_svp)
            d_svp = res['D_alpha']
        dev = self.net.dev
        s_bs = torch.as_tensor(nat.one_electron(0, molecule, basis, svp, self.device), device=dev)
        s_bb = torch.as_tensor(overlap, dtype=torch.float64, device=dev)
        x = torch.linalg.solve(s_bb, s_bs)
        d = x @ torch.as_tensor(d_svp, device=dev) @ x.T
        return self.project(d.cpu().numpy(), overlap, nocc, ortho)

    def predict(self, molecule, basis, sad_density, overlap, nocc, ortho=None):
        import torch
        lay = ClusterLayout(molecule, basis)
        X = (lay.descriptors() - self.mu) / self.sd
        y = self.net.predict_bf16(torch.tensor(X, device=self.net.dev)).cpu().numpy()
        Tsad, _ = lay.local_blocks(sad_density)
        D = lay.assemble(Tsad + y / self.scale)
        return self.project(D, overlap, nocc, ortho)

    def project(self, D, overlap, nocc, ortho=None):
        """Nearest idempotent density with nocc electrons: the nocc natural
        orbitals of largest occupation of D, i.e. the leading eigenvectors of
        X^T S D S X for an orthogonaliser X of the AO basis (X^T S X = 1;
        the SCF driver's canonical X when given, else S^-1/2), so that the
        first-iteration energy is variational."""
        import torch
        dev = self.net.dev
        S = torch.as_tensor(overlap, dtype=torch.float64, device=dev)
        if ortho is None:
            w, u = torch.linalg.eigh(S)
            keep = w > 1.0e-6
            ortho = u[:, keep] / torch.sqrt(w[keep])
        X = torch.as_tensor(ortho, dtype=torch.float64, device=dev)
        Dt = torch.as_tensor(D, dtype=torch.float64, device=dev)
        M = X.T @ S @ Dt @ S @ X
        n, v = torch.linalg.eigh(0.5 * (M + M.T))
        C = X @ v[:, -nocc:]
        return (C @ C.T).cpu().numpy()
