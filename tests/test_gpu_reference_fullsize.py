"""Plain FP64 path against the reference's own CUDA code at the benchmark
sizes.

The reference's unmodified sources (gpu/cuda_kernels/*.cu, built into
oracle/_ref/libnbody_ref.so together with oracle/ref_harness.cu) run one
rebuild + force evaluation in the order of Simulation::rebuildSpatialStructure
and Simulation::computeAccelerations (src/simulation.cpp:137-197, with an
explicit G as tests/integration/cuda/barnes_hut_accuracy_test.cu does), and
export every intermediate.  The library runs the same inputs through nbb_accel
with its export.  Bar: every integer array equal (Morton keys, permutation,
leaf groups, Karras tree, plan, octree topology, leaf ranges, child counts);
every float (box, cell geometry, mass / centre of mass, accelerations) within
1e-12 relative and, on top, bit-identical.

Sizes: Plummer N = 2^20 (theta 0.5, eps 0.01: the headline workload), disk +
bulge N = 2^20 (eps 0.005) and 64 Gaussian blobs N = 2^22 (eps 1e-3), with
the seeds the secondary workloads use; and a 3-step KDK trajectory at
Plummer N = 2^20 against the reference's Simulation::step order
(src/simulation.cpp:100-119).
"""
import numpy as np
import pytest

from test_gpu_parity import FLOAT_RTOL, _compare, _gpu_pipeline
from test_oracle_golden import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build (oracle/_ref/libnbody_ref.so) not present")
    oracle.ref_lib()
    return oracle


def _inputs(recipe, n):
    from nbb import ics

    return {"plummer": lambda: ics.plummer(n, seed=0), "disk": lambda: ics.disk_bulge(n, seed=1),
            "blobs": lambda: ics.blobs(n, seed=2)}[recipe]()


@pytest.mark.parametrize("recipe,n,theta,soft", [
    ("plummer", 1 << 20, 0.5, 0.01),
    ("disk", 1 << 20, 0.5, 0.005),
    ("blobs", 1 << 22, 0.5, 1e-3),
])
def test_pipeline_equals_reference_at_full_size(nbb_mod, reference, recipe, n, theta, soft):
    p = _inputs(recipe, n)
    ref = reference.ref_pipeline(p.mass, p.x, p.y, p.z, theta=theta, soft=soft, g=1.0)
    out, st = _gpu_pipeline(nbb_mod, p, theta, soft, 1.0)
    worst = _compare(out, ref)
    assert max(worst.values()) == 0.0
    assert st.interactions > 0
    # the mixed walk at the same size gives every node the acceptance test:
    # no node is accepted for lack of stack space
    _, _, _, sm = nbb_mod.compute_accelerations(p, theta, soft, 1.0, precision=nbb_mod.PRECISION_MIXED,
                                                stats=True)
    assert sm.interactions > 0 and sm.stack_overflow == 0


def test_trajectory_equals_reference_at_full_size(nbb_mod, reference):
    n, steps, dt, theta, soft = 1 << 20, 3, 1e-3, 0.5, 0.01
    p = _inputs("plummer", n)
    ref = reference.ref_simulate(p, steps, dt, theta, soft, 1.0)
    sim = nbb_mod.Simulation(p, nbb_mod.SimulationConfig(dt, theta, soft, 1.0))
    sim.initialize()
    sim.run(steps)
    got = sim.download() + sim.accelerations()
    for name, a, b in zip(("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"), got, ref):
        assert rel_err(a, b) <= FLOAT_RTOL, name
        assert np.array_equal(a, b), (name, "not bit-identical")
