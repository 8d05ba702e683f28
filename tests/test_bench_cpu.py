"""CPU legs of bench.py: the batched workload's CPU baseline (Triangle's
quality refinement of every domain, one spawned process per host core, domains
assigned by the cost-balanced partition) counts every domain exactly once."""
import os

import pytest

from gpu_cdt_refine_b200 import inputs

TRI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libtriangle_ref.so")


@pytest.mark.skipif(not os.path.exists(TRI), reason="reference Triangle build (make -C oracle ref) not present")
def test_batch_cpu_baseline_counts_every_domain():
    import bench
    from oracle import tri_ref
    doms, thetas = inputs.batch_domains(12, nmax=3000)
    with pytest.raises(RuntimeError):  # workers rebuild the default batch, which these domains are not
        bench.batch_cpu_baseline(doms, thetas, seed=1)
    doms, thetas = inputs.batch_domains(12)
    got = bench.batch_cpu_baseline(doms, thetas)
    want = sum(tri_ref.quality(d, t, 1)[1] for d, t in zip(doms, thetas))
    assert got["output_triangles"] == want
    assert got["value"] > 0 and got["cores"] == min(os.cpu_count() or 1, len(doms))
