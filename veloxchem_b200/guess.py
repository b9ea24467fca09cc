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
atoms' positions in their waters, and radial (and first-moment) neighbour
densities within 5 Angstrom.  The network predicts B_ij - B_ij(SAD) for all
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
NFEAT = NTYPES + 1 + 3 + 3 + 3 + 9 + 3 + 3 + 2 * 2 * len(RBF_CENTERS) + 2 * 3 * len(MOM_CENTERS)

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
    """Atoms, AO lists, water frames and the pair list of one water cluster."""

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
        self.rot = [atom_rotation(self.atom_ls[a], self.frames[self.water[a]].T) for a in range(len(z))]

    def _pairs(self):
        z, xyz = self.z, self.xyz
        n = len(z)
        dist = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2)
        self.dist = dist
        pairs = []
        for i in range(n):
            pairs.append((i, i))
        for i in range(n):
            for j in range(n):
                if i == j or dist[i, j] > PAIR_CUTOFF:
                    continue
                if z[i] == z[j] and j < i:
                    continue
                if z[i] == 1 and z[j] == 8:
                    continue
                pairs.append((i, j))
        self.pairs = np.array(pairs, dtype=np.int64)

    # ---- descriptors
    def _env(self, i):
        """Radial O / H neighbour densities and first moments (local frame) of atom i."""
        d = self.dist[i]
        mask = (d > 1e-8) & (d < ENV_CUTOFF)
        out = []
        for el in (8, 1):
            sel = mask & (self.z == el)
            out.append(np.exp(-((d[sel][:, None] - RBF_CENTERS[None, :]) / RBF_WIDTH) ** 2).sum(axis=0))
        v = (self.xyz[mask] - self.xyz[i]) / d[mask][:, None]
        v = v @ self.frames[self.water[i]]
        g = np.exp(-((d[mask][:, None] - MOM_CENTERS[None, :]) / MOM_WIDTH) ** 2)
        out.append((g[:, :, None] * v[:, None, :]).sum(axis=0).ravel())
        return np.concatenate(out)

    def descriptors(self):
        n = len(self.z)
        env = [self._env(i) for i in range(n)]
        X = np.zeros((len(self.pairs), NFEAT), dtype=np.float32)
        for p, (i, j) in enumerate(self.pairs):
            zi, zj = self.z[i], self.z[j]
            if i == j:
                t = 0 if zi == 8 else 1
            else:
                t = 2 if (zi == 8 and zj == 8) else (3 if zi == 8 else 4)
            wa, wb = self.water[i], self.water[j]
            Fa, Fb = self.frames[wa], self.frames[wb]
            dv = self.xyz[j] - self.xyz[i]
            f = [np.eye(NTYPES)[t], [1.0 if wa == wb else 0.0], [self.dist[i, j], math.exp(-self.dist[i, j]),
                                                                  1.0 / (1.0 + self.dist[i, j])],
                 dv @ Fa, dv @ Fb, (Fa.T @ Fb).ravel(), (self.xyz[i] - self.origin[wa]) @ Fa,
                 (self.xyz[j] - self.origin[wb]) @ Fb, env[i], env[j]]
            X[p] = np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in f])
        return X

    # ---- blocks
    def local_blocks(self, D):
        """Local-frame blocks of D (row-major, padded to NOUT) and their mask."""
        T = np.zeros((len(self.pairs), NOUT), dtype=np.float32)
        M = np.zeros((len(self.pairs), NOUT), dtype=np.float32)
        for p, (i, j) in enumerate(self.pairs):
            blk = self.rot[i] @ D[np.ix_(self.atom_aos[i], self.atom_aos[j])] @ self.rot[j].T
            k = blk.size
            T[p, :k] = blk.ravel()
            M[p, :k] = 1.0
        return T, M

    def assemble(self, B):
        """Global density from local-frame pair blocks (row-major, padded)."""
        D = np.zeros((self.nao, self.nao))
        for p, (i, j) in enumerate(self.pairs):
            ni, nj = len(self.atom_aos[i]), len(self.atom_aos[j])
            blk = self.rot[i].T @ np.asarray(B[p, :ni * nj], dtype=np.float64).reshape(ni, nj) @ self.rot[j]
            D[np.ix_(self.atom_aos[i], self.atom_aos[j])] = blk
            if i != j:
                D[np.ix_(self.atom_aos[j], self.atom_aos[i])] = blk.T
        return 0.5 * (D + D.T)


# ------------------------------------------------------------ the guess driver

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

    def predict(self, molecule, basis, sad_density, overlap, nocc):
        import torch
        lay = ClusterLayout(molecule, basis)
        X = (lay.descriptors() - self.mu) / self.sd
        y = self.net.predict_bf16(torch.tensor(X, device=self.net.dev)).cpu().numpy()
        Tsad, _ = lay.local_blocks(sad_density)
        D = lay.assemble(Tsad + y / self.scale)
        return self.project(D, overlap, nocc)

    def project(self, D, overlap, nocc):
        """Nearest idempotent density with nocc electrons: the nocc natural
        orbitals of largest occupation of D (eigenvectors of S^1/2 D S^1/2),
        so that the first-iteration energy is variational."""
        import torch
        dev = self.net.dev
        S = torch.as_tensor(overlap, dtype=torch.float64, device=dev)
        w, u = torch.linalg.eigh(S)
        keep = w > 1.0e-6
        u, w = u[:, keep], w[keep]
        sh = (u * torch.sqrt(w)) @ u.T
        sih = (u / torch.sqrt(w)) @ u.T
        Dt = torch.as_tensor(D, dtype=torch.float64, device=dev)
        n, v = torch.linalg.eigh(sh @ Dt @ sh)
        C = sih @ v[:, -nocc:]
        return (C @ C.T).cpu().numpy()
