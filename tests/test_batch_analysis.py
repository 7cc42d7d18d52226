"""The batch analysis (baas_analyze_batch) runs stages 2-7 system by system on host threads and
concatenates the results; the schedule must be the one the whole block-diagonal pattern gets in
a single analysis, array for array (every exported field and the final group DAG), on batches of
stencils, variable-coefficient grids and k-NN systems of uneven sizes."""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, BatchSchedule, Schedule, batch_concat, gen
from baas_b200._native import FIELDS, GROUP_DAG_FIELDS

BATCHES = {
    "vardiff": lambda: gen.batch_vardiff2d(nsys=9, kmin=8, kmax=40, seed=2),
    "mixed": lambda: [gen.laplace3d(6, 1e-3), gen.knn_stiffness(nodes=300, k=8, seed=1), gen.laplace2d(17),
                      gen.knn_stiffness(nodes=120, k=6, seed=4), gen.vardiff2d(23, seed=3), gen.laplace2d(1)],
    "two": lambda: [gen.laplace2d(30), gen.laplace3d(9, 1e-3)],
}


@pytest.mark.parametrize("nthread", [1, 8, 16])
@pytest.mark.parametrize("name", list(BATCHES))
def test_batch_analysis_equals_the_whole_pattern(name, nthread):
    systems = BATCHES[name]()
    A, _ = batch_concat(systems)
    whole = Schedule(A, kind=KERNEL_ICCG, nthread=nthread)
    batch = BatchSchedule(systems, nthread=nthread)
    for f in list(FIELDS) + list(GROUP_DAG_FIELDS):
        assert np.array_equal(whole.export(f), batch.export(f)), f"{name} nthread={nthread} field {f}"
