"""Layer stacks the device Green network does not model are refused at the seam: the reference's open bottom and PEC
planes inside the stack (mom25d multilayer.py:96-111) and wideband layers raise NotImplementedError, whether the
stack is this package's LayerStack or an object shaped like the reference's, instead of being solved as a grounded
stack."""
from types import SimpleNamespace

import numpy as np
import pytest

from mom25d_b200 import board as B


def layers():
    return [B.Layer(0.2e-3, 3.5), B.Layer(1.0e-3, 4.4), B.Layer(0.2e-3, 3.5)]


def test_grounded_stacks_are_accepted():
    st = B.LayerStack(layers(), top='open')
    assert st.bottom == 'pec' and st.pec == () and np.allclose(st.z, [0, 0.2e-3, 1.2e-3, 1.4e-3])
    B.LayerStack(layers(), top='pec')


@pytest.mark.parametrize('kw', [dict(bottom='open'), dict(pec=(1,)), dict(bottom='open', bottom_er=2.2, pec=(0, 2))])
def test_open_bottom_and_internal_planes_are_refused(kw):
    with pytest.raises(NotImplementedError):
        B.LayerStack(layers(), **kw)


def test_bad_arguments_stay_value_errors():
    with pytest.raises(ValueError):
        B.LayerStack(layers(), bottom='lid')
    with pytest.raises(ValueError):
        B.LayerStack(layers(), top='lid')


@pytest.mark.parametrize('attrs', [dict(bottom='open', pec=()), dict(bottom='pec', pec=(2,)),
                                   dict(bottom='pec', pec=(), dispersive=True)])
def test_a_reference_shaped_stack_is_refused_by_the_board(attrs):
    st = B.LayerStack(layers())
    foreign = SimpleNamespace(**{**vars(st), **attrs})
    with pytest.raises(NotImplementedError):
        B.Board(foreign, np.zeros((0, 2)), np.zeros((0, 3), int), np.zeros(0, int))
    B.Board(st, np.zeros((0, 2)), np.zeros((0, 3), int), np.zeros(0, int))
