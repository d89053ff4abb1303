# SPDX-License-Identifier: MIT
"""Generate tests/golden/settled_pile_64x32x32.npz: the 65,536-box pile of the
learned-warm-start benchmark (box_pile((64, 32, 32), seed=4)) after 300 ticks
of plain AVBD (legacy profile, 10 sweeps) from its spawn grid, stepped by the
CUDA path. It is the shared starting state of bench.py's GPU and CPU arms.
Run on a GPU host:  python tests/golden/make_settled_pile.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "parallel-mater_b200"))

from pmb200 import core, scenes  # noqa: E402

FRAMES = 300


def main():
    scene = scenes.box_pile((64, 32, 32), seed=4)
    w = core.World(scene)
    for _ in range(FRAMES):
        w.step(stats=False)
    st = w.step()
    states = w.states()
    np.savez_compressed(os.path.join(HERE, "settled_pile_64x32x32.npz"), states=states.view(np.float32).reshape(-1, 13),
                        frames=FRAMES + 1)
    print("saved", scene.n, "bodies; last tick stats", st)


if __name__ == "__main__":
    main()
