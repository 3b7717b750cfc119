"""python -m everest_b200.tmine.single_query <query.yaml>
(the reference's system/single-query.py)."""
import sys

from .frontend import MiningSingle


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 1:
        print("usage: python -m everest_b200.tmine.single_query <query.yaml>", file=sys.stderr)
        return 2
    MiningSingle(argv[0]).run()
    return 0


if __name__ == "__main__":
    sys.exit(main())
