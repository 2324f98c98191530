"""The NIF NxStereo.CudaSegment calls (nif/nx_stereo_cuda_nif.cpp), built
against a fake Erlang runtime (tests/erts_stub) because this image has no
Erlang/OTP: its functions, arities and dirty flags as NxStereo.CudaNif
declares them, its argument checks, and without a device its refusal to
open a context, with the reason."""
import os

import pytest

from tests.erts_stub import harness


@pytest.fixture(scope="module")
def nif():
    return harness.Nif()


def test_the_functions_the_elixir_module_declares(nif):
    assert nif.module == "Elixir.NxStereo.CudaNif"
    declared = open(os.path.join(harness.ROOT, "elixir", "lib", "nx_stereo", "cuda_nif.ex")).read()
    for (name, arity), (_, flags) in nif.funcs.items():
        assert f"def {name}(" in declared
        assert declared.split(f"def {name}(")[1].split(")")[0].count(",") + 1 == arity
    # configure allocates device memory and open creates a context: both dirty
    assert nif.funcs[("open", 1)][1] and nif.funcs[("configure", 2)][1]
    assert not nif.funcs[("run", 5)][1]


def test_bad_arguments_are_badarg(nif):
    assert nif.text(nif.call("open", nif.binary(b"zero"))) == ":badarg"
    assert nif.text(nif.call("configure", nif.lib.fake_int(1), nif.binary(b"\x01"))) == ":badarg"
    assert nif.text(nif.call("run", nif.lib.fake_int(1), nif.binary(b"\x02"), nif.lib.fake_pid(1),
                             nif.lib.fake_ref(1), nif.lib.fake_int(10))) == ":badarg"
    assert nif.text(nif.call("release", nif.lib.fake_int(1), nif.lib.fake_int(1))) == ":badarg"


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="a GPU is present")
def test_without_a_device_open_says_why(nif):
    reply = nif.text(nif.call("open", nif.lib.fake_int(0)))
    assert reply.startswith("{:error, <<") and reply.endswith(">>}")
