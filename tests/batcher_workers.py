"""Worker functions for the AsyncBatcher tests (importable by spawned pool workers)."""
import os
import time


def square_after(i, delay):
    """i * i after `delay` seconds (later tasks may finish first)."""
    time.sleep(delay)
    return i * i, os.getpid()


def fail_on(i, bad):
    if i == bad:
        raise ValueError(f"task {i} failed")
    return i


def shared_sum(name, size, k):
    """Sum of the shared array's first k entries, read in the worker."""
    from cupyram_b200 import AsyncBatcher
    obj = AsyncBatcher.load_shared_object(name, size)
    return float(obj["a"][:k].sum())


def pack_batch(args, kw):
    """CPU preparation of a march batch in a worker (the intended use: the main
    process only uploads and marches)."""
    from cupyram_b200 import batch as B
    envs, p, zs, zr, pr = B.prepare(*args, dict(kw))
    return B.build_batch(envs, p, zs, zr, pr, False)
