"""Error paths of the C ABI: status codes instead of the reference's blocking cin.get()."""
import numpy as np
import pytest

from conftest import get_case

pytestmark = pytest.mark.gpu


def test_inverted_element_is_rejected():
    from cfdv_b200 import gpu as G, meshgen as mg
    case = mg.lid(4)
    el = case.elements.copy()
    el[5, :4] = el[5, [1, 0, 3, 2]]  # mirror one element
    bad = mg.Case("bad", 2, case.nodes, el, case.control, case.aero)
    with pytest.raises(G.CfdvError) as e:
        G.FDVSolver(bad)
    assert e.value.code == 3


def test_out_of_order_calls():
    from cfdv_b200 import gpu as G
    with G.FDVSolver(get_case("lid8")) as s:
        s.load_node_records()
        with pytest.raises(G.CfdvError) as e:
            s.gmres()
        assert e.value.code == 6
        with pytest.raises(G.CfdvError) as e:
            s.set_state(np.zeros(3))
        assert e.value.code == 1


def test_non_finite_state_reports_status():
    from cfdv_b200 import gpu as G
    case = get_case("lid8")
    with G.FDVSolver(case) as s:
        s.load_node_records()
        U = s.get_state()
        U[10] = np.nan
        s.set_state(U)
        with pytest.raises(G.CfdvError) as e:
            s.form(1e-3)
        assert e.value.code == 4
        # the context stays usable after the error
        s.load_node_records()
        s.form(1e-3)
