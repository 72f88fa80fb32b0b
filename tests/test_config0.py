"""The sensitivity record of the small discharge (tests/golden/config0_sensitivity.json,
made by tests/golden/make_config0.py): the restated loop against itself started
from a density changed by a relative 1e-12.  Up to step 100 (the first microwave
update) the two runs agree far below 1e-8 -- the window in which
tests/test_config0_gpu.py compares the device with the restated loop at 1e-8;
50 steps later Te differs by more than 1e-6 and by step 1000 the runs are
unrelated, so no comparison at 1e-8 exists there."""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("phi", "rhoe", "rhoi", "Te")


def test_the_loop_amplifies_small_differences_after_the_heating():
    with open(os.path.join(HERE, "golden", "config0_sensitivity.json")) as f:
        s = json.load(f)["steps"]
    assert max(s["100"][k] for k in FIELDS) < 1e-10         # the window the device test uses
    assert s["150"]["Te"] > 1e-6                            # 1e-12 grown by 1e6 and more in 50 steps
    assert min(s["1000"][k] for k in FIELDS) > 1e-2         # no comparison exists at step 1000
