"""``AsyncBatcher``: host-side prefetch of batch preparation.

Same interface as the reference's ``cupyram/batching.py:5-152``: an iterator of
argument tuples is mapped through a picklable worker function in a process
pool, ``max_prefetch`` results are kept in flight, and results are yielded in
submission order so the main process can feed the GPU engine while the next
batches are prepared.  ``share_object`` / ``load_shared_object`` /
``cleanup_shared_object`` hand large read-only inputs to the workers through
POSIX shared memory instead of pickling them per task.

The pool uses the ``spawn`` start method: a worker forked from a process that
already holds a CUDA context can hang.
"""
import multiprocessing as mp
import pickle
from concurrent.futures import ProcessPoolExecutor
from multiprocessing import shared_memory


class AsyncBatcher:
    def __init__(self, input_data_iterator, worker_func, max_prefetch=1, max_workers=2):
        if max_prefetch < 1 or max_workers < 1:
            raise ValueError("max_prefetch and max_workers must be >= 1")
        self.input_iter = iter(input_data_iterator)
        self.worker_func = worker_func
        self.max_prefetch = max_prefetch
        self.max_workers = max_workers
        self._pending = []
        self._executor = None

    def __iter__(self):
        ctx = mp.get_context("spawn")
        with ProcessPoolExecutor(max_workers=self.max_workers, mp_context=ctx) as ex:
            self._executor = ex
            for _ in range(self.max_prefetch):
                self._submit()
            while self._pending:
                fut = self._pending.pop(0)
                res = fut.result()
                self._submit()
                yield res
        self._executor = None

    def _submit(self):
        try:
            args = next(self.input_iter)
        except StopIteration:
            return
        self._pending.append(self._executor.submit(self.worker_func, *args))

    @staticmethod
    def share_object(obj):
        data = pickle.dumps(obj, protocol=pickle.HIGHEST_PROTOCOL)
        shm = shared_memory.SharedMemory(create=True, size=len(data))
        shm.buf[:len(data)] = data
        name, size = shm.name, len(data)
        shm.close()
        return name, size

    @staticmethod
    def load_shared_object(name, size):
        shm = shared_memory.SharedMemory(name=name)
        try:
            return pickle.loads(bytes(shm.buf[:size]))
        finally:
            shm.close()

    @staticmethod
    def cleanup_shared_object(name):
        try:
            shm = shared_memory.SharedMemory(name=name)
        except FileNotFoundError:
            return
        shm.close()
        shm.unlink()
