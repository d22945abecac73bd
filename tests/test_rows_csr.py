"""Host-side row definitions: branch-id lists to the trip CSR the session
takes (duplicates dropped, first occurrence kept), on vectorised paths that
keep the CSR as the only copy."""

import numpy as np

from gpusim2grid_b200.batch import _rows_csr


def test_single_branch_rows_keep_only_the_csr():
    rows, ptr, ids = _rows_csr([[3], [5], [3]])
    assert rows is None
    assert ptr.tolist() == [0, 1, 2, 3] and ids.tolist() == [3, 5, 3]
    assert ptr.dtype == np.int32 and ids.dtype == np.int32
    rows, ptr, ids = _rows_csr(np.array([[7], [2]]))
    assert rows is None and ptr.tolist() == [0, 1, 2] and ids.tolist() == [7, 2]


def test_other_rows_drop_duplicates_in_order():
    rows, ptr, ids = _rows_csr([[4, 2, 4], [], [1]])
    assert rows is None
    assert ptr.tolist() == [0, 2, 2, 3] and ids.tolist() == [4, 2, 1]


def test_vectorised_rows_equal_the_per_row_reference():
    """The flattened conversion of general rows (any count per row,
    repeats, negative ids left for the library to reject) equals the
    per-row one: first occurrences in row order."""
    rng = np.random.default_rng(1)
    for _ in range(200):
        rows = [[int(x) for x in rng.integers(-3, 20, int(rng.integers(0, 6)))]
                for _ in range(int(rng.integers(2, 40)))]
        rows[0] = rows[0] + [7, 7]  # not every row of one id
        ref = [list(dict.fromkeys(r)) for r in rows]
        _, ptr, ids = _rows_csr(rows)
        assert ptr.tolist() == np.cumsum([0] + [len(r) for r in ref]).tolist()
        assert ids.tolist() == [v for r in ref for v in r]
    _, ptr, ids = _rows_csr(np.array([[1, 2], [2, 2]]))
    assert ptr.tolist() == [0, 2, 3] and ids.tolist() == [1, 2, 2]
