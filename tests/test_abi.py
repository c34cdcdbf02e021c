"""The C ABI: the library loads without a GPU and exports every function the
public headers (include/*.h) declare; the Python binding knows each of them."""
import re
from pathlib import Path

import restir_b200 as rb

INCLUDE = Path(__file__).resolve().parent.parent / "include"
DECLARATION = re.compile(r"^[A-Za-z_][\w \t\*]*?\b(restir_\w+)\s*\(", re.M)


def declared() -> dict[str, list[str]]:
    names = {}
    for header in sorted(INCLUDE.glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))
        found = sorted(set(DECLARATION.findall(text)))
        if found:
            names[header.name] = found
    return names


def test_headers_declare_the_passes():
    names = declared()
    assert {"restir_gpu.h", "restir_frame.h", "restir_host.h", "restir_cache.h", "restir_display.h"} <= set(names)
    assert "restir_gi_temporal" in names["restir_gpu.h"]
    assert "restir_taa" in names["restir_display.h"]


def test_library_exports_every_declared_function():
    lib = rb.load()
    missing = [(h, n) for h, fns in declared().items() for n in fns if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_has_a_signature_for_every_declared_function():
    known = set(rb._SIGNATURES)
    missing = [(h, n) for h, fns in declared().items() for n in fns if n not in known]
    assert not missing, missing


def test_struct_layouts_match_the_binding():
    import ctypes as C

    from restir_b200 import abi
    lib = rb.load()
    structs = {name: obj for name, obj in vars(abi).items()
               if name.startswith("Restir") and isinstance(obj, type) and issubclass(obj, C.Structure)}
    assert len(structs) >= 19
    for name, cls in structs.items():
        assert lib.restir_struct_size(name.encode()) == C.sizeof(cls), name
    assert lib.restir_struct_size(b"NoSuchStruct") == 0


def test_fp64_passes_refuse_images_beyond_32_bit_pixel_counts():
    """restir_reference_accumulate and restir_error count pixels in 32 bits:
    a 65536 x 65536 image is refused before anything is launched (no device
    memory is touched, so this runs without a GPU)."""
    import ctypes as C

    from restir_b200.abi import RestirParams
    lib = rb.load()
    p = RestirParams()
    p.width, p.height = 65536, 65536
    fake = C.c_void_p(256)
    assert lib.restir_reference_accumulate(p, fake, fake, fake, 0, None) == rb.ERROR_TOO_LARGE
    assert lib.restir_error(p, fake, fake, fake, fake, fake, None) == rb.ERROR_TOO_LARGE
