"""Restart files on the CPU: the run configuration survives the archive's
JSON metadata unchanged, and a file of another format is refused before
any device work."""
import json

import numpy as np
import pytest

from helpers import setup_for
from piernik_b200 import restart
from piernik_b200.config import BND_OUT, BND_PER


@pytest.mark.parametrize("s", [
    setup_for("mhd", n=(24, 20, 16), lim="moncen", cflcontrol="redo"),
    setup_for("hd", n=(32, 16, 1), bnd=((BND_OUT, BND_OUT), (BND_PER, BND_PER), (BND_PER, BND_PER))),
    setup_for("mhd", n=(8, 8, 8), lim="weno3", solver="unsplit", ord_mag_prolong=-4).replace(
        fluids=[("ion", 5.0 / 3.0), ("neu", 1.4), ("dst", -1.0)]),
])
def test_setup_round_trip(s):
    back = restart._setup_from(json.loads(json.dumps(restart._setup_dict(s))))
    assert back == s and back.dl == s.dl and back.ext == s.ext and back.nvar == s.nvar


def test_other_format_refused(tmp_path):
    path = str(tmp_path / "old.npz")
    np.savez(path, meta=np.array(json.dumps({"format": restart.FORMAT + 1})))
    with pytest.raises(ValueError, match="restart format"):
        restart.load(path)
