"""Angular-block matrices with the reference's storage semantics.

Mirrors ``CMatrix`` / ``CSubMatrix`` / ``CMatrices`` and ``make_matrix``
(src/math/Matrix.cpp, SubMatrix.cpp, Matrices.cpp, MatrixFunc.cpp:36-59) as the
Python tests of the reference use them:

* a symmetric matrix stores only angular blocks (i, j) with i <= j; ``set_values``
  copies those blocks from a dense array (src/python/ExportMath.cpp:258-276) and
  ``full_matrix`` mirrors off-diagonal blocks (Matrix.cpp:348-373);
* a general matrix stores all blocks;
* ``SubMatrix ==`` compares elementwise with rtol = atol = 1e-12
  (SubMatrix.cpp:105-115, MathFunc.hpp:74-77).
"""

import enum

import numpy as np


class mat_t(enum.Enum):
    symmetric = 0
    antisymmetric = 1
    general = 2


def _equal(a, b, rtol=1.0e-12, atol=1.0e-12):
    a = np.asarray(a)
    b = np.asarray(b)
    return bool(np.all(np.abs(a - b) < np.maximum(atol, rtol * np.maximum(np.abs(a), np.abs(b)))))


class SubMatrix:
    """A dense block with row/column offsets: dims = [row0, col0, nrows, ncols]."""

    def __init__(self, dims=None, values=None):
        dims = [0, 0, 0, 0] if dims is None else [int(v) for v in dims]
        self._dims = dims
        self._values = np.zeros((dims[2], dims[3])) if values is None else \
            np.array(values, dtype=np.float64).reshape(dims[2], dims[3])

    def set_values(self, values):
        self._values[:, :] = np.asarray(values, dtype=np.float64)

    def get_dimensions(self):
        return list(self._dims)

    def to_numpy(self):
        return self._values.copy()

    def number_of_rows(self):
        return self._dims[2]

    def number_of_columns(self):
        return self._dims[3]

    def at(self, i, j):
        return self._values[i, j]

    def symmetrize(self):
        if self._dims[2] == self._dims[3]:
            self._values = self._values + self._values.T

    def __eq__(self, other):
        return self._dims == other._dims and _equal(self._values, other._values)

    def __ne__(self, other):
        return not self.__eq__(other)


class Matrix:
    """Angular-block matrix over a molecular basis (reference CMatrix)."""

    def __init__(self, blocks=None, mtype=mat_t.general):
        self._blocks = {} if blocks is None else dict(blocks)
        self._type = mtype

    # --- construction -------------------------------------------------------
    def add(self, submat, angpair):
        if isinstance(submat, SubMatrix):
            self._blocks[tuple(angpair)] = submat
        else:
            self._blocks[tuple(angpair)] = SubMatrix(submat)

    def set_type(self, mtype):
        self._type = mtype

    def get_type(self):
        return self._type

    def angular_pairs(self):
        return sorted(self._blocks.keys())

    def submatrix(self, angpair):
        return self._blocks.get(tuple(angpair), SubMatrix())

    def is_angular_order(self, angpair):
        return tuple(angpair) in self._blocks

    def number_of_rows(self):
        return max((b._dims[0] + b._dims[2] for b in self._blocks.values()), default=0)

    def number_of_columns(self):
        return max((b._dims[1] + b._dims[3] for b in self._blocks.values()), default=0)

    # --- values -------------------------------------------------------------
    def zero(self):
        for b in self._blocks.values():
            b._values[:, :] = 0.0

    def scale(self, factor):
        for b in self._blocks.values():
            b._values *= factor

    def set_values(self, values):
        values = np.asarray(values, dtype=np.float64)
        if values.ndim != 2 or values.shape != (self.number_of_rows(), self.number_of_columns()):
            return
        for b in self._blocks.values():
            r0, c0, nr, nc = b._dims
            b._values[:, :] = values[r0:r0 + nr, c0:c0 + nc]

    def symmetrize(self):
        if self._type == mat_t.symmetric:
            for (i, j), b in self._blocks.items():
                if i == j:
                    b.symmetrize()

    def full_matrix(self):
        nr, nc = self.number_of_rows(), self.number_of_columns()
        full = np.zeros((nr, nc))
        for (i, j), b in self._blocks.items():
            r0, c0, n0, n1 = b._dims
            full[r0:r0 + n0, c0:c0 + n1] = b._values
            if i != j and self._type == mat_t.symmetric:
                full[c0:c0 + n1, r0:r0 + n0] = b._values.T
            if i != j and self._type == mat_t.antisymmetric:
                full[c0:c0 + n1, r0:r0 + n0] = -b._values.T
        return SubMatrix([0, 0, nr, nc], full)

    def to_numpy(self):
        return self.full_matrix().to_numpy()

    def __eq__(self, other):
        if self._type != other._type or self.angular_pairs() != other.angular_pairs():
            return False
        return all(self._blocks[k] == other._blocks[k] for k in self._blocks)

    def __ne__(self, other):
        return not self.__eq__(other)

    def __add__(self, other):
        out = Matrix({k: SubMatrix(b._dims, b._values + other._blocks[k]._values)
                      for k, b in self._blocks.items()}, self._type)
        return out

    def copy(self):
        return Matrix({k: SubMatrix(b._dims, b._values) for k, b in self._blocks.items()}, self._type)

    def __copy__(self):
        return self.copy()

    def __deepcopy__(self, memo):
        return self.copy()


def make_matrix(basis, mtype):
    """Angular-block layout of a basis (reference matfunc::make_matrix)."""
    lmax = basis.max_angular_momentum()
    offs = basis.angular_offsets()
    sizes = [basis.number_of_basis_functions(l) * (2 * l + 1) for l in range(lmax + 1)]
    mat = Matrix(mtype=mtype)
    for i in range(lmax + 1):
        for j in range(lmax + 1):
            if mtype in (mat_t.symmetric, mat_t.antisymmetric) and j < i:
                continue
            mat.add(SubMatrix([offs[i], offs[j], sizes[i], sizes[j]]), (i, j))
    return mat


class Matrices:
    """Keyed collection of matrices (reference CMatrices, keys sorted as strings)."""

    def __init__(self):
        self._mats = {}

    def add(self, matrix, key):
        self._mats[str(key)] = matrix.copy()

    def matrix(self, key):
        return self._mats.get(str(key))

    def keys(self):
        return sorted(self._mats.keys())

    def number_of_matrices(self):
        return len(self._mats)

    def zero(self):
        for m in self._mats.values():
            m.zero()

    def symmetrize(self):
        for m in self._mats.values():
            m.symmetrize()
