"""Multi-GPU partitioning of NPROMA blocks.

Columns are independent in CLOUDSC (the only dependency is the vertical
recurrence, cloudsc.F90:1219-4128), so G GPUs take contiguous block ranges
[g*N/G, (g+1)*N/G) and run with no exchange on the data path; only scalar
statistics (step times, warning counts) are reduced across ranks.
"""


def block_range(ngpblks, rank, world):
    """[first, last) block indices owned by ``rank`` of ``world``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return (rank * ngpblks) // world, ((rank + 1) * ngpblks) // world
