"""Host logic of the eager FheBool / FheUint8 front end (no GPU): the circuit
each operator runs, the global server key and the thread-local division flag
(shortint/mod.rs:10-56, bool/mp_api.rs:136-145 / 183-185)."""
import threading

import pytest

from conftest import pz


def fhe():
    import importlib
    return importlib.import_module("phantom-zone_b200.fhe")


# operator -> (input ciphertexts, output ciphertexts)
SHAPES = {
    "and": (2, 1), "nand": (2, 1), "or": (2, 1), "nor": (2, 1), "xor": (2, 1), "xnor": (2, 1),
    "add": (16, 8), "sub": (16, 8), "mul": (16, 8),
    "overflowing_add": (16, 9), "overflowing_sub": (16, 9),
    "div": (16, 9), "div_or": (17, 9), "rem": (16, 8), "div_rem": (16, 17), "div_rem_or": (17, 17),
    "eq": (16, 1), "neq": (16, 1), "lt": (16, 1), "gt": (16, 1), "le": (16, 1), "ge": (16, 1),
    "mux": (17, 8), "max": (16, 8), "min": (16, 8),
}


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_operator_circuit_shapes(name):
    c = fhe()._build(name)
    info = c.info()
    assert (info["inputs"], info["outputs"]) == SHAPES[name]
    assert info["gates"] > 0


def test_division_circuits_share_gates_with_and_without_previous_flag():
    """div_or = div + one OR of the previous flag (shortint/mod.rs:42-56)."""
    F = fhe()
    assert F._build("div_or").info()["gates"] == F._build("div").info()["gates"] + 1
    assert F._build("div_rem_or").info()["gates"] == F._build("div_rem").info()["gates"] + 1
    # remainder alone does not evaluate is_zero(divisor)
    assert F._build("rem").info()["gates"] < F._build("div_rem").info()["gates"]


def test_server_key_set_once():
    F = fhe()
    F.clear_server_key()
    with pytest.raises(RuntimeError, match="Server key not set"):
        F._server()
    F.set_server_key("engine", "key")
    try:
        with pytest.raises(RuntimeError, match="twice"):
            F.set_server_key("engine2", "key2")
        assert F._server() == ("engine", "key")
    finally:
        F.clear_server_key()


def test_div_zero_flag_thread_local_and_reset():
    F = fhe()
    F.reset_error_flags()
    assert F.div_zero_error_flag() is None
    F._TLS.div_zero = "flag"
    seen = []
    t = threading.Thread(target=lambda: seen.append(F.div_zero_error_flag()))
    t.start()
    t.join()
    assert seen == [None]
    assert F.div_zero_error_flag() == "flag"
    F.reset_error_flags()
    assert F.div_zero_error_flag() is None


def test_package_exports_value_api():
    P = pz()
    for name in ["FheBool", "FheUint8", "set_server_key", "div_zero_error_flag", "reset_error_flags"]:
        assert hasattr(P, name)
