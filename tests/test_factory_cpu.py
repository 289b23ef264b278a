"""index_factory's grammar against the reference's (index_factory.cpp:63-153):
for each description, the same index type (fourcc) or the same exception
class as the reference compiled from its sources (oracle/_ref), where a
std::invalid_argument surfaces as ValueError and a std::out_of_range from
an oversized number as IndexError (swignsparse.swig:47-59)."""

import ctypes

import pytest

import nsparse
import oracle as O

ERRORS = {1: "ValueError", 2: "RuntimeError", 3: "IndexError", 4: "MemoryError"}
SPECS = [
    "brutal", "inverted", "seismic", "seismic_sq", "idmap,brutal", "idmap,seismic,lambda=5",
    "idmap", "idmap,", "", "nonsense", "seismic,lambda=abc", "seismic,lambda=99999999999",
    "seismic,lambda=7|beta=3|alpha=0.3|seed=1", "seismic,alpha=x",
    "seismic_sq,quantizer=16bit|vmin=0|vmax=2", "seismic_sq,quantizer=4bit",
    "seismic_sq,quantizer=8bit|vmin=a", "seismic,unknown=3", "seismic,lambda", "seismic,lambda=3=4",
    "brutal,lambda=3", "BRUTAL", " brutal", "brutal ", "seismic,lambda=-5", "seismic,lambda= 4",
    "seismic,seed=-1", "seismic,lambda=1e3", "seismic,alpha=1e-1", "idmap,idmap,brutal",
    "seismic_sq,vmin=2|vmax=1", "seismic,", "seismic,|", "seismic,lambda=4|",
    "seismic,lambda=4||beta=2", "idmap,seismic_sq,quantizer=16bit", "inverted,x",
    "seismic,lambda=4,beta=2", "seismic;lambda=4", "seismic,alpha=nan", "seismic,alpha=inf",
    "seismic,seed=4294967296", "seismic,beta=0", "seismic,lambda=0", "seismic_sq,quantizer=",
    "idmap,nonsense",
]


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("spec", SPECS)
def test_factory_agrees_with_reference(spec):
    try:
        ours = nsparse.index_factory(16, spec).id()
    except Exception as e:  # noqa: BLE001 -- the class is the result
        ours = type(e).__name__
    L = O.ref_lib("generic")
    buf = ctypes.create_string_buffer(4)
    rc = L.ref_factory_status(16, spec.encode(), buf)
    ref = buf.raw.decode() if rc == 0 else ERRORS[rc]
    assert ours == ref
