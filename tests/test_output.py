"""Host-side output writers that need no GPU (dl_write_pvd)."""
import xml.etree.ElementTree as ET

from dynlattice_b200.engine import write_pvd


def test_pvd_collection(tmp_path):
    """ParaViewModule's collection file: one DataSet per output with its time
    and the file name relative to the collection (ParaViewModule.cpp:186-216)."""
    path = tmp_path / "visual" / "step.pvd"
    write_pvd(path, [0.0, 0.01, 0.02], ["step0.vtu", "step1.vtu", "step2.vtu"])
    root = ET.parse(path).getroot()
    assert root.get("type") == "Collection"
    ds = root.findall("Collection/DataSet")
    assert [d.get("file") for d in ds] == ["step0.vtu", "step1.vtu", "step2.vtu"]
    assert [float(d.get("timestep")) for d in ds] == [0.0, 0.01, 0.02]
    assert all(d.get("part") == "0" and d.get("group") == "" for d in ds)
