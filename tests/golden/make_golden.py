"""Extract the reference's golden vectors for the elasticity hot path into tests/golden/.

The reference ships MATLAB-exported JSON fixtures (written by its tests/export_rust_*.m scripts)
that its Rust tests compare against:

* rust/tests/fixtures/iga_kernel.json        -> iga_kernel.json  (rust/tests/iga_vs_matlab.rs:22-73)
* rust/tests/fixtures/immersed_tilted_box.json -> immersed_tilted_box.json
                                                (rust/tests/immersed_vs_matlab.rs:20-73)
* rust/tests/fixtures/topopt3d_8x4x2.json    -> topopt3d_8x4x2.json (rust/tests/topopt_vs_matlab.rs:15-40)

The reference tree is only mounted in the build container, so the vectors are copied here (the
fields the tests read, values unchanged) and committed.  Run:

    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import sys

FILES = {
    "iga_kernel.json": None,  # every field is used
    "immersed_tilted_box.json": None,
    "topopt3d_8x4x2.json": None,
}


def main(ref_root: str) -> None:
    src_dir = os.path.join(ref_root, "rust", "tests", "fixtures")
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, keep in FILES.items():
        with open(os.path.join(src_dir, name)) as f:
            data = json.load(f)
        if keep is not None:
            data = {k: data[k] for k in keep}
        with open(os.path.join(out_dir, name), "w") as f:
            json.dump(data, f, separators=(",", ":"))
        print(f"wrote {name}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout root>")
    main(sys.argv[1])
