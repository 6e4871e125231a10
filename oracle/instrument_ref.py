"""TEST INFRASTRUCTURE (build step of oracle/Makefile).

Writes a copy of the reference's sequential SOSP update
(src/sequentialSOSPUpdate.cu of SMShovan/MOSP-CUDA) into oracle/_ref/ with
two clock reads added, so that the benchmark's reference arm can report the
compute-only time of the reference's own CPU update next to its whole
file-API call. The copy is generated at build time from the sources where
they lie and is not committed. Nothing else in the function changes:

  * mark 1 before the section banner of its Phase 1 (src/sequentialSOSPUpdate.cu:456):
    the text input has been read and the batch applied;
  * mark 2 before the section banner of its output stage (:614): the
    update has been computed, the text output follows.

Usage: python instrument_ref.py <reference src/sequentialSOSPUpdate.cu> <out.cu>
"""
import re
import sys


def main():
    src, out = sys.argv[1], sys.argv[2]
    lines = open(src).read().split("\n")
    banner = re.compile(r"^\s*// =+$")

    def banner_before(label):
        # the banner block is "// ===", "// <label>", "// ===": return the
        # index of its first line
        for i in range(1, len(lines) - 1):
            if label in lines[i] and banner.match(lines[i - 1]) and banner.match(lines[i + 1]):
                return i - 1
        raise SystemExit(f"instrument_ref.py: section '{label}' not found in {src}")

    first = banner_before("PHASE 1")
    second = banner_before("WRITE OUTPUT")
    if not first < second:
        raise SystemExit("instrument_ref.py: unexpected section order")
    indent = re.match(r"^(\s*)", lines[first]).group(1)
    lines.insert(second, f"{indent}mosp_ref_phase_mark(2);")
    lines.insert(first, f"{indent}mosp_ref_phase_mark(1);")
    lines.insert(0, 'extern "C" void mosp_ref_phase_mark(int which);')
    with open(out, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
