"""Generate tests/golden/struct_layout.json from the REFERENCE's own header.

Compiles a small C program against the reference's src/util/basic_types.h
(read in place under the reference root, with the configure-time
tblis_config.h that oracle/build_ref.sh writes into oracle/_ref/gen) and
records sizeof / alignof / offsetof of tblis_tensor and tblis_matrix and the
type_t values, as the reference's C ABI lays them out.  tests/test_capi.py
compares this library's include/tblis_stra_b200.h against the fixture, so the
comparison needs neither the reference nor its build on the machine that runs
the tests.

Usage: python tests/golden/make_layout.py [REFERENCE_ROOT]
(run oracle/build_ref.sh first; default root: $TBLIS_STRA_REFERENCE_ROOT,
else a directory named "reference" beside this repository).
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

# The program prints one JSON object; the same source is compiled against the
# library's header by tests/test_capi.py (LAYOUT_SOURCE).
LAYOUT_SOURCE = r"""
#include <stdio.h>
#include <stddef.h>
#include HEADER
#define F(S, f) printf("\"%s.%s\": [%zu, %zu], ", #S, #f, offsetof(S, f), sizeof(((S*)0)->f))
int main(void)
{
    printf("{");
    F(tblis_tensor, type); F(tblis_tensor, conj); F(tblis_tensor, scalar); F(tblis_tensor, data);
    F(tblis_tensor, ndim); F(tblis_tensor, len); F(tblis_tensor, stride);
    F(tblis_matrix, type); F(tblis_matrix, conj); F(tblis_matrix, scalar); F(tblis_matrix, data);
    F(tblis_matrix, m); F(tblis_matrix, n); F(tblis_matrix, rs); F(tblis_matrix, cs);
    printf("\"sizeof.tblis_tensor\": %zu, \"alignof.tblis_tensor\": %zu, ",
           sizeof(tblis_tensor), _Alignof(tblis_tensor));
    printf("\"sizeof.tblis_matrix\": %zu, \"alignof.tblis_matrix\": %zu, ",
           sizeof(tblis_matrix), _Alignof(tblis_matrix));
    printf("\"sizeof.len_type\": %zu, \"sizeof.stride_type\": %zu, \"sizeof.label_type\": %zu, ",
           sizeof(len_type), sizeof(stride_type), sizeof(label_type));
    printf("\"TYPE_SINGLE\": %d, \"TYPE_FLOAT\": %d, \"TYPE_DOUBLE\": %d, \"TYPE_SCOMPLEX\": %d, "
           "\"TYPE_DCOMPLEX\": %d}\n", (int)TYPE_SINGLE, (int)TYPE_FLOAT, (int)TYPE_DOUBLE,
           (int)TYPE_SCOMPLEX, (int)TYPE_DCOMPLEX);
    return 0;
}
"""


def layout(include_flags, header) -> dict:
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        with open(src, "w") as f:
            f.write(LAYOUT_SOURCE)
        subprocess.check_call(["gcc", "-std=gnu11", "-w", f"-DHEADER=\"{header}\""] + include_flags
                              + [src, "-o", exe])
        return json.loads(subprocess.check_output([exe]).decode())


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "TBLIS_STRA_REFERENCE_ROOT", os.path.join(os.path.dirname(REPO), "reference"))
    gen = os.path.join(REPO, "oracle", "_ref", "gen")
    if not os.path.isfile(os.path.join(gen, "tblis_config.h")):
        sys.exit("run oracle/build_ref.sh first (it writes oracle/_ref/gen/tblis_config.h)")
    flags = ["-I" + os.path.join(gen, "cfgdir"), "-I" + gen, "-I" + os.path.join(ref, "src", "util")]
    out = layout(flags, os.path.join(ref, "src", "util", "basic_types.h"))
    out["_source"] = "reference src/util/basic_types.h:52-63,264-272,341-352 compiled as C (gcc, x86-64)"
    with open(os.path.join(HERE, "struct_layout.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps(out, sort_keys=True))


if __name__ == "__main__":
    main()
