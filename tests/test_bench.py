"""Host logic of bench.py that needs no GPU: the committed DRAM-traffic table the roofline reads."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_table_rows():
    """Every row of profiles/traffic.tsv parses to (bytes per launch, capture iterations or None);
    the persistent solve's rows carry the Krylov iteration count of their capture, since the
    bench scales a solve's traffic by its own iterations per launch."""
    tr = _bench().load_traffic()
    assert ("bicgstab_persistent", "large_slab") in tr
    for (kernel, workload), (nbytes, iters) in tr.items():
        assert nbytes > 0, (kernel, workload)
        assert iters is None or iters > 0
    assert tr[("bicgstab_persistent", "large_slab")][1] is not None
    assert tr[("element_assemble", "large_slab")][1] is None
