import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # Host-only helpers build with gcc in seconds; the CUDA library and the
    # reference harness are built by __graft_entry__.build() (nvcc).
    import oracle
    from cublox_b200 import synth

    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build(ref=False)
    synth.build()
