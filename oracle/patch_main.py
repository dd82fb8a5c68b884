"""oracle/patch_main.py -- TEST INFRASTRUCTURE ONLY (a build step).

Writes a copy of the reference's src/main.cpp whose time-evolution loop
(main.cpp:274-288, the `for (int it = 1; it <= nt; it++)` block) is replaced
by the GPU loop of coolbubble_b200/binding/cb_main_loop.hpp, included just
before main(). Everything else of the file is kept as it is. The copy goes to
the build folder (oracle/_ref), never into the repository.

  python3 patch_main.py <reference src/main.cpp> <output .cpp>
"""
import sys

LOOP_HEAD = "for (int it = 1; it <= nt; it++)"
MAIN_HEAD = "int main(int argc, const char *argv[])"
CALL = "    if (cb_main_loop(s, folder, snapshotSteps, trackWall, progressEvery) != 0) return 1;  /* coolbubble_b200 */\n"
INCLUDE = '#include "cb_main_loop.hpp"  /* coolbubble_b200: the time loop on the GPU */\n'


def patch(lines):
    heads = [i for i, ln in enumerate(lines) if LOOP_HEAD in ln]
    mains = [i for i, ln in enumerate(lines) if ln.strip() == MAIN_HEAD]
    if len(heads) != 1 or len(mains) != 1:
        raise SystemExit("patch_main.py: expected one time loop and one main() (found %d, %d)"
                         % (len(heads), len(mains)))
    start = heads[0]
    depth, end, opened = 0, None, False
    for i in range(start, len(lines)):
        for ch in lines[i]:
            if ch == "{":
                depth += 1
                opened = True
            elif ch == "}":
                depth -= 1
                if opened and depth == 0:
                    end = i
                    break
        if end is not None:
            break
    if end is None:
        raise SystemExit("patch_main.py: the time loop's closing brace was not found")
    return lines[:mains[0]] + [INCLUDE, "\n"] + lines[mains[0]:start] + [CALL] + lines[end + 1:]


def main():
    src, dst = sys.argv[1], sys.argv[2]
    with open(src) as f:
        lines = f.readlines()
    with open(dst, "w") as f:
        f.writelines(patch(lines))


if __name__ == "__main__":
    main()
