"""Host-side stream handles of MDSystem.set_stream: torch gives its default
stream the handle 0, which the C ABI reads as "the library's own stream", so
the Python mirror passes cudaStreamLegacy for it (work on the system is then
ordered with torch's default-stream work).  Checked without a GPU by
intercepting the ABI call."""
import ctypes as C

import pytest


def test_default_stream_handle_maps_to_legacy(monkeypatch):
    pytest.importorskip("torch")
    import mdforce.core as core
    seen = []

    def fake(h, stream):
        seen.append(stream.value)
        return 0

    monkeypatch.setattr(core.lib, "md_system_set_stream", fake)

    class Dummy:
        h = C.c_void_p(1234)

    core.MDSystem.set_stream(Dummy(), 0)
    core.MDSystem.set_stream(Dummy(), None)
    core.MDSystem.set_stream(Dummy(), 0x7f00deadbeef)
    assert seen == [core.CUDA_STREAM_LEGACY, None, 0x7f00deadbeef]
