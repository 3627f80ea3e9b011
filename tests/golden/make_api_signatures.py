"""Writes api_signatures.json: the parameter lists (name, kind, default) of the
reference's public functions on the rasterization path, read by importing the
reference package on the CPU (textured_gaussians/rendering.py and
textured_gaussians/cuda/_wrapper.py; importing them needs no GPU), and the keys
of the ``meta`` dict each renderer returns (read from its source).

Run from the repository root with the reference checkout as the argument:

    python tests/golden/make_api_signatures.py <path to the textured_gaussians checkout>
"""
import inspect
import json
import os
import sys

FUNCTIONS = {
    "textured_gaussians.rendering": ["rasterization_textured_gaussians", "rasterization_2dgs"],
    "textured_gaussians.cuda._wrapper": [
        "spherical_harmonics", "fully_fused_projection_2dgs", "isect_tiles", "isect_offset_encode",
        "rasterize_to_pixels_textured_gaussians", "rasterize_to_pixels_2dgs", "generate_mipmap",
        "selective_adam_update",
    ],
}


def describe(fn):
    out = []
    for p in inspect.signature(fn).parameters.values():
        out.append({"name": p.name, "kind": p.kind.name,
                    "default": None if p.default is inspect.Parameter.empty else repr(p.default)})
    return out


def meta_keys(fn):
    """Keys of the last ``meta = {...}`` dict literal in the function's source (the renderers' ``meta``)."""
    import ast
    import textwrap
    tree = ast.parse(textwrap.dedent(inspect.getsource(fn)))
    keys = None
    for node in ast.walk(tree):
        if (isinstance(node, ast.Assign) and isinstance(node.value, ast.Dict)
                and any(isinstance(t, ast.Name) and t.id == "meta" for t in node.targets)):
            keys = [k.value for k in node.value.keys]
    return keys


def main(ref_root):
    sys.path.insert(0, ref_root)
    import importlib
    table = {}
    for mod, names in FUNCTIONS.items():
        m = importlib.import_module(mod)
        for n in names:
            if hasattr(m, n):
                table[f"{mod}.{n}"] = describe(getattr(m, n))
    rendering = importlib.import_module("textured_gaussians.rendering")
    for n in FUNCTIONS["textured_gaussians.rendering"]:
        table[f"meta_keys:{n}"] = meta_keys(getattr(rendering, n))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "api_signatures.json"), "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
        f.write("\n")
    print(f"{len(table)} entries written")


if __name__ == "__main__":
    main(sys.argv[1])
