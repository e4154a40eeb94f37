"""The multigrid levels' coefficient arrays ``aw ... ap`` (read by the
reference's own harness, tests/test_mg.py:16-32) equal the arrays the
reference's ``_mgcoeff`` kernel writes (multigrid.py:23-67), bit for bit,
on every level, at the harness spacing and at a different spacing per
axis.  The golden arrays come from running the reference source
(tests/golden/make_golden.py).  The views need no GPU."""
from types import SimpleNamespace

import numpy as np
import pytest

from helpers import golden

NAMES = ("aw", "ae", "as_", "an", "ab", "at", "ap")


@pytest.mark.parametrize("tag,h0", [("coef", (1 / 16,) * 3), ("coefx", (0.1, 0.2, 0.3))])
def test_coefficient_views_match_reference(tag, h0):
    from warpflow.multigrid import _CoeffView
    g = golden("mg16_l3")
    for l in range(3):
        n = 16 >> l
        s = 2.0 ** l
        lev = SimpleNamespace(n3=(n,) * 3, shape=(n + 2,) * 3, h=tuple(x * s for x in h0))
        for name in NAMES:
            got = _CoeffView(lev, name).numpy()
            np.testing.assert_array_equal(got, g["%s%d_%s" % (tag, l, name)],
                                          err_msg="%s level %d %s" % (tag, l, name))
