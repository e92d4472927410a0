"""The vertical solve's own check (thorx_check_thomas): the reference's optional diagnostic
DIAG_CHECK_THOR_VERTICAL_INT_THOMAS_RESULT (src/headers/dyn/thor_vertical_int.h:486-523) flags any
interior interface whose tridiagonal residual exceeds 1e-8 of the right-hand side. After steps of
the Held-Suarez state in both forms and with the vertical options the reference varies
(non-hydrostatic or not, deep or shallow, gravity varying with height), no interface may be
flagged."""
import pytest

import thor_b200
from thorx_testlib import RefGrid, grid_dict, initial_state, make_params, thorx_params

GLEVEL, NV, DT = 4, 24, 1200.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("over", [dict(), dict(NonHydro=0), dict(DeepModel=0),
                                  dict(GravHeightVar=1)])
def test_thomas_residual_below_the_reference_epsilon(precision, over):
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT, **over)
    st = initial_state(g.arrays, g.point_num, NV, c, amp=1.0)
    x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT, precision=precision))
    for k, v in st.items():
        x.set(k, v)
    for _ in range(3):
        x.step(2)
        worst, nbad = x.check_thomas(1e-8)
        assert nbad == 0 and worst < 1e-8, (worst, nbad)
        assert worst > 0.0  # the check sees the system (an all-zero residual would mean no rows)
    x.close(), g.close()
