"""CPU tests of the drop-in boundary: the library loads, exports every symbol
the public headers declare, and its host-only entry points behave like the
reference's.  No device work runs here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "parode_b200", "libParODEShared.so")


def _declared_functions():
    names = set()
    pat = re.compile(r"^\s*(?:C_EXPORT\s+)?(?:void|int|long long|ParODE_Plan\s*\*)\s+([A-Za-z_][A-Za-z0-9_]*)\s*\(")
    for fn in ("ParODECInterface.h", "parode_ext.h"):
        with open(os.path.join(INCLUDE, fn)) as fh:
            for line in fh:
                m = pat.match(line)
                if m:
                    names.add(m.group(1))
    return names


def test_headers_declare_reference_abi():
    names = _declared_functions()
    ref = {"GetErrorDescription", "InitializeAllGPUs", "GetAvailableGPUs", "GetDeviceName", "InitializeSelectedGPUs",
           "SimulateODE", "RegisterInput", "CloseGPUC", "StartTimer", "StopTimer"}
    assert ref <= names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build first: make -C parode_b200"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = _declared_functions() - exported
    assert not missing, missing
    lib = ctypes.CDLL(LIB)
    for name in _declared_functions():
        getattr(lib, name)


def test_c_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "use.c"
    src.write_text("#include <ParODECInterface.h>\n#include <parode_ext.h>\n#include <ParODEEnums.h>\n"
                   "int main(void){ int e=0; char b[256]; GetErrorDescription(&e, b); return (int)ParODE_NumOutputs(0,0,1,1) == 2 ? 0 : 1; }\n")
    subprocess.run(["gcc", "-DC_INCLUDE", "-I", INCLUDE, "-c", str(src), "-o", str(tmp_path / "use.o")], check=True)
    cpp = tmp_path / "use.cpp"
    cpp.write_text("#include <ParODECppInterface.h>\nint main(){ matrixf A(2,2,0.0f); vectorf x(2, 1.0f);\n"
                   " std::string s; GetErrorDescription(ParODE_NoGPU, s); return (int)A.size1() - 2 + (int)x.size() - 2; }\n")
    exe = tmp_path / "usecpp"
    subprocess.run(["g++", "-std=c++11", "-I", INCLUDE, str(cpp), "-o", str(exe), f"-L{os.path.dirname(LIB)}",
                    "-lParODEShared", f"-Wl,-rpath,{os.path.dirname(LIB)}"], check=True)
    subprocess.run([str(exe)], check=True)


def test_host_entry_points():
    import parode_b200 as pb

    assert pb.error_description(0) == "No Error"
    assert "initialized" in pb.error_description(-2)
    assert pb.error_description(12345) == "Unknown Error"
    # step-count rule of the reference (floating truncation included)
    assert pb.num_outputs(0, 0.0, 99 * 0.1, 0.1) == 100
    assert pb.num_outputs(1, 0.0, 99 * 0.1, 0.1) == 99
    assert pb.num_outputs(0, 1.0, 0.0, 0.1) == -1



def test_executions_option_round_trip():
    import parode_b200 as pb

    assert pb.get_option(pb.OPT_EXECUTIONS) == 1
    pb.set_option(pb.OPT_EXECUTIONS, 16)
    assert pb.get_option(pb.OPT_EXECUTIONS) == 16
    with pytest.raises(pb.ParODEError):
        pb.set_option(pb.OPT_EXECUTIONS, 0)
    assert pb.get_option(pb.OPT_EXECUTIONS) == 16
    pb.set_option(pb.OPT_EXECUTIONS, 1)


def test_fault_injection_options_round_trip():
    import parode_b200 as pb

    assert pb.get_option(pb.OPT_FAULT_ALLOC) == -1
    pb.set_option(pb.OPT_FAULT_ALLOC, 3)
    assert pb.get_option(pb.OPT_FAULT_ALLOC) == 3
    with pytest.raises(pb.ParODEError):
        pb.set_option(pb.OPT_FAULT_ALLOC, -2)
    pb.set_option(pb.OPT_FAULT_ALLOC, -1)
    assert pb.get_option(pb.OPT_FAULT_WITHHOLD) == 0
    pb.set_option(pb.OPT_FAULT_WITHHOLD, 1)
    assert pb.get_option(pb.OPT_FAULT_WITHHOLD) == 1
    pb.set_option(pb.OPT_FAULT_WITHHOLD, 0)


def test_pool_keep_option():
    """A negative byte count is refused; the value reads back as last set."""
    import parode_b200 as pb

    keep = pb.get_option(pb.OPT_POOL_KEEP)
    assert keep >= 0
    with pytest.raises(pb.ParODEError):
        pb.set_option(pb.OPT_POOL_KEEP, -1)
    assert pb.get_option(pb.OPT_POOL_KEEP) == keep


def test_discretise_option_round_trip():
    import parode_b200 as pb

    assert pb.get_option(pb.OPT_DISCRETISE) == pb.DISCRETISE_AUTO
    pb.set_option(pb.OPT_DISCRETISE, pb.DISCRETISE_HOST)
    assert pb.get_option(pb.OPT_DISCRETISE) == pb.DISCRETISE_HOST
    with pytest.raises(pb.ParODEError):
        pb.set_option(pb.OPT_DISCRETISE, 3)
    assert pb.get_option(pb.OPT_DISCRETISE) == pb.DISCRETISE_HOST
    pb.set_option(pb.OPT_DISCRETISE, pb.DISCRETISE_AUTO)


def test_tuning_file_round_trip(tmp_path):
    """Entries of one GPU survive save and load; other GPUs' lines are skipped."""
    import parode_b200 as pb

    src = tmp_path / "tune.txt"
    src.write_text("NVIDIA_B200 0 64 8 8 20 1 5 0.25\nNVIDIA_B200 1 128 2 2 16 0 3 1.5\n"
                   "Other_GPU 0 64 8 8 20 1 6 0.2\nbad line\n")
    pb.tune_clear()
    assert pb.tune_load(str(src), gpu="NVIDIA B200") == 2
    out = tmp_path / "out.txt"
    assert pb.tune_save(str(out), gpu="NVIDIA B200") == 2
    lines = sorted(out.read_text().split("\n"))
    assert [ln.split()[:8] for ln in lines if ln] == [
        ["NVIDIA_B200", "0", "64", "8", "8", "20", "1", "5"], ["NVIDIA_B200", "1", "128", "2", "2", "16", "0", "3"]]
    pb.tune_clear()
    assert pb.tune_save(str(out), gpu="NVIDIA B200") == 0


def test_not_initialised_errors():
    import parode_b200 as pb

    pb.close()
    with pytest.raises(pb.ParODEError) as ei:
        pb.simulate(np.eye(2), None, None, None, np.ones(2), 0, 0.0, 1.0, 0.1)
    assert ei.value.code == -2
    t, y, e = pb.simulate_f32(np.eye(2), None, None, None, np.ones(2), 0, 0.0, 1.0, 0.1)
    assert e == -2


def test_python_module_surface():
    import ParODE

    for name in ("GetErrorDescription", "InitializeAllGPUs", "GetAvailableGPUs", "GetDeviceName",
                 "InitializeSelectedGPUs", "SimulateODE", "RegisterInput", "CloseGPU", "StartTimer", "StopTimer"):
        assert callable(getattr(ParODE, name))
    assert issubclass(ParODE.error, Exception)
    assert ParODE.GetErrorDescription(-1).startswith("Sorry, no GPU")
    # invalid matrices return None, as the reference module does
    assert ParODE.SimulateODE([[1.0, 2.0]], [], [], [], 0, 0.0, 0.1, 10, [1.0], 0) is None
