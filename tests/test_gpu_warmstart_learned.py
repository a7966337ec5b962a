"""What the trained warm-start network gains: on held-out synthetic holograms
(seeds outside the training set), FISTA started from the network's x0 reaches
plain FISTA's 100-iteration objective (within 1e-3) in fewer iterations than
plain FISTA from zero, which stays the reference.  Uses the committed weights
(trained by ``warmstart.py train``)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_network_reaches_the_objective_in_fewer_iterations(rihvr):
    import importlib

    ws = importlib.import_module(rihvr.__name__ + ".warmstart")
    if not os.path.exists(ws.WEIGHTS):
        pytest.fail(f"trained weights missing: {ws.WEIGHTS}")
    seeds = np.arange(200_000, 200_006)
    with rihvr.UNet(ws.PLANES, ws.SIZE, ws.SIZE) as net:
        net.load(ws.WEIGHTS)
        rows = ws.evaluate(net, seeds)
    s = ws.summary(rows)
    print(s)
    assert s["reached_warm"] == len(rows)  # every warm start reaches the target
    assert s["mean_iters_warm"] < s["mean_iters_plain"]
    # the untrained network gives no such gain: the learning is what helps
    with rihvr.UNet(ws.PLANES, ws.SIZE, ws.SIZE, seed=5) as raw:
        base = ws.summary(ws.evaluate(raw, seeds))
    print("untrained", base)
    assert s["mean_iters_warm"] < base["mean_iters_warm"]
