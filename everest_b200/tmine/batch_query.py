"""python -m everest_b200.tmine.batch_query <graph> <gpu> <query-dir>
(the reference's system/batch-query.py): every YAML in the directory, in
name order, against one loaded graph."""
import os
import sys

from . import locations
from .frontend import Mining


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 3:
        print("usage: python -m everest_b200.tmine.batch_query <graph> <gpu> <query-dir>", file=sys.stderr)
        return 2
    graph, gpu, qdir = argv
    if not os.path.exists(graph):
        graph = os.path.join(locations.inputGraphRoot(), graph)
    m = Mining(graph, int(gpu))
    for q in sorted(os.listdir(qdir)):
        if not q.endswith((".yaml", ".yml")):
            continue
        print("@@@ [output starts]")
        print(f"# process {q}")
        print("@@@ [output ends]")
        m.run(os.path.join(qdir, q))
    return 0


if __name__ == "__main__":
    sys.exit(main())
