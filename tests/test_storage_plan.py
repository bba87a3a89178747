"""The device storage each matrix gets (fb_matrix_storage_plan, host only): diagonal storage for
structured grids numbered lexicographically, sliced / uniform ELL with int16 column offsets
otherwise, absolute columns for the rectangular transfer matrices; the layout the solver actually
uploads is the same function of the same inputs."""
import numpy as np

from featb200 import assembly as AS
from featb200.lafem import SparseMatrixCSR


def _csr(m):
    return SparseMatrixCSR.from_scipy(m.tocsr())


def test_lexicographic_grids_take_diagonal_storage(featlib):
    fb = featlib
    A2 = AS.stiffness(6, 2)
    p = fb.storage_plan(_csr(A2), AS.boundary_dofs(6, 2))
    assert p["kind"] == "diagonal" and p["diagonals"] == 9 and p["width"] == 9
    assert p["entries"] == ((A2.shape[0] + 31) // 32) * 32 * 9
    A3 = AS.stiffness(3, 3)
    p3 = fb.storage_plan(_csr(A3), AS.boundary_dofs(3, 3))
    assert p3["kind"] == "diagonal" and p3["diagonals"] == 27
    # 3D level 4: 4,913 rows, 31% of them Dirichlet rows (stored empty): diagonal storage would pad
    # more than 12.5%, so the level stays in ELL
    assert fb.storage_plan(_csr(AS.stiffness(4, 3)), AS.boundary_dofs(4, 3))["kind"] != "diagonal"
    # switched off: uniform ELL with row-relative int16 columns
    q = fb.storage_plan(_csr(A2), AS.boundary_dofs(6, 2), diagonal=False)
    assert q["kind"] == "ell" and q["narrow"] and q["width"] == 9
    # small levels take it whatever their padding (the Dirichlet rows of level 2 are 64% of the rows)
    assert fb.storage_plan(_csr(AS.stiffness(2, 2)), AS.boundary_dofs(2, 2))["kind"] == "diagonal"


def test_other_numberings_and_shapes(featlib):
    fb = featlib
    from helpers import load_golden, to_lafem_levels
    lv = to_lafem_levels(load_golden("c1_L4")["levels"])
    # the reference's own refinement numbering: far more than 27 column offsets
    p = fb.storage_plan(lv[0]["matrix"], lv[0]["filter"].indices)
    assert p["kind"] != "diagonal" and p["narrow"]
    # reverse Cuthill-McKee of a lexicographic grid: offsets vary from row to row
    A = AS.stiffness(6, 2)
    assert fb.storage_plan(_csr(A), AS.boundary_dofs(6, 2), ordering="rcm")["kind"] != "diagonal"
    # the prolongation is rectangular: absolute columns, never diagonal
    P = fb.storage_plan(_csr(AS.prolongation(6, 2)))
    assert P["kind"] != "diagonal" and not P["narrow"] and P["width"] == 4


def test_unsorted_row_keeps_the_stored_order(featlib):
    """A row whose columns are not increasing cannot be summed in stored order along ascending
    diagonals: it stays in ELL."""
    fb = featlib
    A = AS.stiffness(4, 2).tocsr()
    rp, ci, v = A.indptr.copy(), A.indices.copy(), A.data.copy()
    r = 40
    ci[rp[r]], ci[rp[r] + 1] = ci[rp[r] + 1], ci[rp[r]]
    v[rp[r]], v[rp[r] + 1] = v[rp[r] + 1], v[rp[r]]
    M = SparseMatrixCSR(rp, ci, v, A.shape)
    assert fb.storage_plan(M)["kind"] != "diagonal"
    assert fb.storage_plan(_csr(A))["kind"] == "diagonal"
