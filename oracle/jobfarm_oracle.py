"""The reference's leader job loop, restated (test infrastructure).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the job farm in
t2-relion_b200/parallel.py.  The shipped library never uses it.

`Leader.request(follower)` is one pass of the leader's loop in MlOptimiserMpi::expectation
(src/ml_optimiser_mpi.cpp:1140-1302) for a job request from MPI rank `follower` (1-based):
the random subset of the follower (odd ranks subset 1), the next range of that subset
(guided chunks when the halves are split and a half has several followers), the reply
(-1, -1) once the subset is done, and the counters updated by JOB_NPAR, including the
reference's count of 1 for a done reply (JOB_LAST - JOB_FIRST + 1 with both -1).  The path
without subset_size and without the debugging cap (xjl_type) is restated.
"""


class Leader:
    def __init__(self, n_half1, n_particles, nr_followers, nr_pool, split_halves=True):
        self.n1, self.n = n_half1, n_particles
        self.size = nr_followers + 1          # MPI processes: leader + followers
        self.nr_pool = nr_pool
        self.split = split_halves
        self.done = 0
        self.done_h = {1: 0, 2: 0}

    def request(self, follower):
        if self.split:
            half = 1 if follower % 2 == 1 else 2
            process_num = (self.size - 1) // 2
            if half == 1:
                first_h, last_h = 0, self.n1 - 1
            else:
                first_h, last_h = self.n1, self.n - 1
            my_done = self.done_h[half]
            todo = last_h - first_h + 1
            job_first = first_h + my_done
            if process_num == 1:
                job_last = last_h
            else:
                chunk = (todo - my_done + 2 * process_num - 1) // (2 * process_num)
                chunk = max(self.nr_pool, chunk)
                job_last = min(last_h, job_first + chunk - 1)
        else:
            half = 0
            my_done = self.done
            todo = self.n
            job_first = self.done
            job_last = min(self.n - 1, job_first + self.nr_pool - 1)
        if my_done >= todo:
            job_first = job_last = -1
        npar = job_last - job_first + 1
        self.done += npar
        if self.split:
            self.done_h[half] += npar
        return None if job_first < 0 else (job_first, job_last)
