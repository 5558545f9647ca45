"""Write tests/golden/reference_kats.json: the known answers of the reference's
own test suite for this path, plus one oracle regression value.

Sources (read as text; the reference is MATLAB and cannot run here):
  Runtime/tests/test_runtime.m:179-184  wust_ncg_direction cases
  Runtime/tests/test_runtime.m:22-28,185-188  projection of 1500 m/s by a
      crossing direction with alpha 1 -> 1512 m/s inside the mask
When the reference tree is present, the script checks that each literal
still appears in test_runtime.m before writing.  The tree's location is the
first command-line argument, else the WUST_REFERENCE_ROOT environment
variable, else /root/reference.

The stencil_opt_params entry is an oracle regression value (no reference
output exists for it); it guards the restatement against drift.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

REF_ROOT = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WUST_REFERENCE_ROOT", "/root/reference"))
REF_TEST = os.path.join(REF_ROOT, "Runtime", "tests", "test_runtime.m")

NCG = [
    # [d, beta, gz] = wust_ncg_direction([1; 2], [2; 1], [1; .5], 1.5, [-1; -2], true)
    dict(g=[1, 2], z=[2, 1], prev_z=[1, .5], prev_gz=1.5, previous_direction=[-1, -2], same_frequency=True,
         beta=4 / 3, gz=4.0, source="test_runtime.m:179-180"),
    # restart on non-descent
    dict(g=[1, 2], z=[2, 1], prev_z=[1, .5], prev_gz=1.5, previous_direction=[100, 100], same_frequency=True,
         beta=0.0, direction=[-2, -1], source="test_runtime.m:181-182"),
    # frequency change restarts CG
    dict(g=[1, 2], z=[2, 1], prev_z=[1, .5], prev_gz=1.5, previous_direction=[-1, -2], same_frequency=False,
         beta=0.0, source="test_runtime.m:183-184"),
]
PROJECTION = dict(initial=1500.0, alpha=1.0, step_damping=0.25, max_update_mps=12.0, bounds_mps=[1300.0, 1800.0],
                  projected=1512.0, source="test_runtime.m:22-28,185-188")
LITERALS = [r"wust_ncg_direction\(\[1; 2\], \[2; 1\], \[1; \.5\], 1\.5, \[-1; -2\], true\)",
            r"abs\(beta - 4 / 3\) < 1e-14 && gz == 4",
            r"isequal\(d, \[-2; -1\]\)",
            r"updated\(mask\) == 1512",
            r"'step_damping', \.25, 'max_update_mps', 12, 'bounds_mps', \[1300, 1800\]"]


def main():
    if os.path.exists(REF_TEST):
        text = open(REF_TEST).read()
        for lit in LITERALS:
            if not re.search(lit, text):
                raise SystemExit(f"literal not found in test_runtime.m: {lit}")
    from oracle.helmholtz_fp64 import stencil_opt_params
    args = [1400.0, 1700.0, 1e5, 1e-3, 1.0]
    b, d, e = stencil_opt_params(*args)
    out = dict(ncg_direction=NCG, projection=PROJECTION,
               stencil_opt_params=dict(args=args, b=b, d=d, e=e, source="oracle regression"))
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
