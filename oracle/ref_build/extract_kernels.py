"""Oracle pin build helper: copies the named __global__ / __device__ /
HD_INLINE / HOST_DEVICE functions of a reference source file (verbatim, in file order)
into an include file under oracle/_ref/, and member-function templates
named Class::member (from their "template <...>" line). Used for files
whose other code does not build on the host (curand initial conditions,
kernel launches, device arrays)."""
import re
import sys


def extract(src, names):
    text = open(src).read()
    lines = text.splitlines(keepends=True)
    out = []
    i = 0
    while i < len(lines):
        line = lines[i]
        # a definition starts with a qualifier line followed by "name(" or
        # with "qualifier type name(" on one line
        head = "".join(lines[i:i + 2])
        m = re.match(r"\s*(__global__|__device__|HD_INLINE|HOST_DEVICE)\b[^\n]*\n?\s*([A-Za-z_]\w*)\s*\(",
                     head)
        head3 = "".join(lines[i:i + 3])
        mt = re.match(r"\s*template\s*<[^>]*>\s*\n\s*\w+\s*\n\s*([A-Za-z_]\w*::[A-Za-z_]\w*)\s*\(",
                      head3)
        if (m and m.group(2) in names) or (mt and mt.group(1) in names):
            depth, j, started = 0, i, False
            while j < len(lines):
                code = lines[j].split("//", 1)[0]  # braces in comments do not count
                depth += code.count("{") - code.count("}")
                started = started or "{" in code
                out.append(lines[j])
                j += 1
                if started and depth == 0:
                    break
            i = j
            continue
        i += 1
    return "".join(out)


if __name__ == "__main__":
    src, dst, names = sys.argv[1], sys.argv[2], set(sys.argv[3:])
    body = extract(src, names)
    found = set(re.findall(r"(" + "|".join(re.escape(n) for n in names) + r")\s*\(", body))
    missing = names - found
    if missing:
        sys.exit(f"not found in {src}: {sorted(missing)}")
    open(dst, "w").write(body)
