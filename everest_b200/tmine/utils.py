"""Helpers of the reference's system/tmine/utils.py and KernelGen.InspectMotif."""
import re


def libFileToLibName(filename: str) -> str:
    """lib<NAME>.so -> NAME."""
    m = re.match(r".*lib(\w+)\.so$", filename)
    if not m:
        raise ValueError(f"not a plugin library name: {filename}")
    return m.group(1)


def libNameToLibFile(name: str) -> str:
    return "lib" + name + ".so"


def InspectMotif(pathToMotif: str):
    """(mapped nodes before each edge j >= 1, max stack level k - 2, k), as
    the reference's KernelGen.InspectMotif (system/tmine/KernelGen.py:13-29)."""
    mnode, mnode_p = [], []
    allE = 0
    with open(pathToMotif) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            allE += 1
            u, v = parts[0], parts[1]
            mnode_p.append(len(mnode))
            if u not in mnode:
                mnode.append(u)
            if v not in mnode:
                mnode.append(v)
    return mnode_p[1:], allE - 2, allE
