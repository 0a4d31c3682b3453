"""The C ABI's records against the reference's own contract headers: the
header include/re_b200.h is compiled beside contracts/GpuRecordsAbiV1.hpp,
SceneAbiV0.hpp, rt/gpu/CanonicalTraversalScene.hpp,
rt/software_gpu/SoftwareGpu.hpp and integrators/megakernel/MegakernelBridge.hpp
in oracle/ref_abi.cpp, which static_asserts the size, alignment and offset
of every member of every record read or written as-is (a mismatch fails the
oracle/_ref build), and the mirrored enumerations."""
import ctypes as C

import pytest


def test_records_match_reference_contracts(oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    lib = C.CDLL(str(oracle.REF_LIB))
    # 11 records (size + alignment) and 67 members.
    assert lib.ref_abi_checked_fields() == 78
