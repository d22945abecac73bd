"""Host-side row definitions: branch-id lists to the trip CSR the session
takes (duplicates dropped, first occurrence kept; single-branch rows take a
vectorised path that keeps the CSR as the only copy)."""

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
    assert rows == [[4, 2], [], [1]]
    assert ptr.tolist() == [0, 2, 2, 3] and ids.tolist() == [4, 2, 1]
