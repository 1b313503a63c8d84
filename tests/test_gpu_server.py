"""Job server (gpt_server_*): jobs rendered together over resident scenes must give, bit for bit,
the images the frame renderer (gpt_render_frame) gives for the same scene, camera and settings,
whether a job runs alone, mixed with others, one at a time, or through a tiny path pool."""
import time

import numpy as np
import pytest

import pathtracer
import scenes

pytestmark = pytest.mark.gpu

BUDGET = 2 << 30


def no_light_scene():
    s = scenes.cornell_all_models(1)
    mats = s.materials.copy()
    for m in range(len(mats)):
        if mats[m]["model"] == 5:
            mats[m]["model"] = 1
    return scenes.Scene(s.positions, s.normals, s.tangents, s.uvs, s.material_ids, mats, name="cornell-dark",
                        camera=s.camera)


@pytest.fixture(scope="module")
def resident(scene_factory):
    names = ["cornell-all", "cornell-textured", "spheres-small"]
    return {n: scene_factory(n) for n in names} | {"cornell-dark": no_light_scene()}


@pytest.fixture(scope="module")
def frame_renderers(resident):
    out = {}
    for name, s in resident.items():
        r = pathtracer.Renderer(0)
        r.upload_scene(s)
        out[name] = r
    yield out
    for r in out.values():
        r.close()


def frame_reference(renderers, name, scene, w, h, spp, depth, nee, rng_offset=0):
    r = renderers[name]
    cam = scenes.scene_camera(scene, w, h)
    r.render_frame(cam, w, h, spp, depth, nee, rng_offset=rng_offset)
    return r.framebuffer().reshape(-1), r.accumulation().reshape(-1, 4)


def make_server(resident, **kw):
    srv = pathtracer.Server(0, hbm_budget_bytes=kw.pop("hbm_budget_bytes", BUDGET), **kw)
    ids = {name: srv.add_scene(s) for name, s in resident.items()}
    return srv, ids


JOBS = [
    # scene, width, height, spp, depth, nee, rng offset
    ("cornell-all", 40, 30, 4, 6, True, 0),
    ("cornell-all", 33, 17, 16, 8, False, 0),
    ("cornell-textured", 48, 48, 4, 5, True, 0),
    ("cornell-textured", 20, 36, 9, 7, False, 77),
    ("spheres-small", 64, 40, 4, 12, True, 0),
    ("spheres-small", 31, 29, 1, 10, True, 5),
    ("cornell-dark", 24, 24, 4, 6, True, 0),
    ("cornell-all", 96, 64, 2, 8, True, 1000),
]


def check_job(srv, jid, renderers, resident, job):
    name, w, h, spp, depth, nee, off = job
    st = srv.wait(jid, 300)
    assert st["state"] == "done", (job, st, srv.last_error())
    fb, acc = srv.result(jid, accumulation=True)
    ref_fb, ref_acc = frame_reference(renderers, name, resident[name], w, h, spp, depth, nee, off)
    assert np.array_equal(acc.view(np.uint32), ref_acc.view(np.uint32)), job
    assert np.array_equal(fb, ref_fb), job


def submit(srv, ids, resident, job):
    name, w, h, spp, depth, nee, off = job
    cam = scenes.scene_camera(resident[name], w, h)
    return srv.submit(ids[name], cam, w, h, spp, depth, nee, rng_offset=off, keep_accumulation=True)


def test_single_jobs_match_frame_renderer(resident, frame_renderers):
    srv, ids = make_server(resident, pool_size=1 << 16)
    try:
        for job in JOBS:
            check_job(srv, submit(srv, ids, resident, job), frame_renderers, resident, job)
    finally:
        srv.close()


def test_mixed_jobs_match_alone(resident, frame_renderers):
    srv, ids = make_server(resident, pool_size=1 << 18)
    try:
        jids = [submit(srv, ids, resident, job) for job in JOBS]
        for jid, job in zip(jids, JOBS):
            check_job(srv, jid, frame_renderers, resident, job)
        st = srv.stats()
        assert st["completed_jobs"] == len(JOBS)
        expected = sum(w * h * int(np.sqrt(spp)) ** 2 for _, w, h, spp, _, _, _ in JOBS)
        assert st["samples"] == expected
        assert st["admitted_bytes"] == 0
        assert 0 < st["admitted_high_water"] <= BUDGET
    finally:
        srv.close()


def test_host_loop_slices_match_frame_renderer(resident, frame_renderers):
    """Slices whose iterations the host launches one by one (GPT_LOOP_HOST, the mode profilers can
    see) give the same images as the graph slices, i.e. the frame renderer's."""
    srv, ids = make_server(resident, pool_size=1 << 16)
    try:
        srv.set_loop_mode(pathtracer.LOOP_HOST)
        jids = [submit(srv, ids, resident, job) for job in JOBS]
        for jid, job in zip(jids, JOBS):
            check_job(srv, jid, frame_renderers, resident, job)
        srv.set_loop_mode(pathtracer.LOOP_GRAPH)
        check_job(srv, submit(srv, ids, resident, JOBS[0]), frame_renderers, resident, JOBS[0])
        with pytest.raises(pathtracer.GptError):
            srv.set_loop_mode(7)
    finally:
        srv.close()


@pytest.mark.parametrize("schedule", [pathtracer.SCHEDULE_SHORTEST_FIRST, pathtracer.SCHEDULE_OLDEST_FIRST,
                                      pathtracer.SCHEDULE_DEADLINE, pathtracer.SCHEDULE_TWO_CLASS])
def test_schedule_orders_completion_not_images(resident, frame_renderers, schedule):
    """Shortest-first hands idle slots to the job with the fewest samples left, earliest-deadline
    first to the job whose deadline (submit time + slowdown x its size / rate) comes first, and the
    two-class order to short jobs (both are short here) by samples left: in all three, a small job
    submitted right after a large one finishes first. Every policy gives the same images."""
    srv, ids = make_server(resident, pool_size=4096, schedule=schedule)
    try:
        big = ("spheres-small", 128, 128, 64, 12, True, 0)
        small = ("cornell-all", 16, 16, 1, 6, True, 0)
        j_big = submit(srv, ids, resident, big)
        j_small = submit(srv, ids, resident, small)
        check_job(srv, j_small, frame_renderers, resident, small)
        check_job(srv, j_big, frame_renderers, resident, big)
        if schedule != pathtracer.SCHEDULE_OLDEST_FIRST:
            assert srv.poll(j_small)["done_s"] < srv.poll(j_big)["done_s"]
    finally:
        srv.close()
    with pytest.raises(pathtracer.GptError):
        pathtracer.Server(0, schedule=5)


def test_two_class_schedule_keeps_long_jobs_in_submission_order(resident, frame_renderers):
    """Two classes: a short job (render time alone below short_job_seconds) passes the long jobs, and
    the long jobs keep their submission order although the later one has fewer samples left, which
    shortest-first would run first."""
    srv, ids = make_server(resident, pool_size=4096, schedule=pathtracer.SCHEDULE_TWO_CLASS, short_job_seconds=1e-5)
    try:
        long_a = ("spheres-small", 128, 128, 16, 10, True, 0)   # 262,144 paths
        long_b = ("spheres-small", 64, 64, 16, 10, True, 0)     # 65,536 paths
        small = ("cornell-all", 16, 16, 1, 6, True, 0)          # 256 paths
        j_a = submit(srv, ids, resident, long_a)
        j_b = submit(srv, ids, resident, long_b)
        j_s = submit(srv, ids, resident, small)
        for j, job in ((j_a, long_a), (j_b, long_b), (j_s, small)):
            check_job(srv, j, frame_renderers, resident, job)
        done = {j: srv.poll(j)["done_s"] for j in (j_a, j_b, j_s)}
        assert done[j_s] < done[j_a] < done[j_b]
    finally:
        srv.close()


def test_two_class_admission_keeps_room_for_short_jobs(resident, frame_renderers):
    """Two classes under a tight budget: with one long job admitted and the next long job waiting for
    memory, a short job submitted after both is admitted at once from the eighth of the budget that
    long jobs leave free, instead of queueing behind the waiting long job. The long jobs keep their
    order, and every image equals the frame renderer's."""
    # about 1.25 MB for a long job (64 B x 4096 in-flight paths, a ring of 2 passes of 16,384 pixels,
    # accumulator and framebuffer), 30 kB for the short one: one long job fits in 7/8 of the budget, two do not
    budget = 1_450_000
    srv, ids = make_server(resident, pool_size=4096, schedule=pathtracer.SCHEDULE_TWO_CLASS, short_job_seconds=1e-5,
                           hbm_budget_bytes=budget)
    try:
        long_job = ("spheres-small", 128, 128, 16, 10, True, 0)   # 262,144 paths
        small = ("cornell-all", 16, 16, 1, 6, True, 0)            # 256 paths
        j_a = submit(srv, ids, resident, long_job)
        j_b = submit(srv, ids, resident, long_job)
        j_s = submit(srv, ids, resident, small)
        for j, job in ((j_a, long_job), (j_b, long_job), (j_s, small)):
            check_job(srv, j, frame_renderers, resident, job)
        done = {j: srv.poll(j)["done_s"] for j in (j_a, j_b, j_s)}
        assert done[j_s] < done[j_a] < done[j_b]
        assert srv.poll(j_s)["admit_s"] < srv.poll(j_b)["admit_s"]
        assert srv.stats()["admitted_high_water"] <= budget
    finally:
        srv.close()


def test_deadline_schedule_does_not_pass_over_a_late_job(resident, frame_renderers):
    """With a deadline of one render time (slowdown 1), a large job that has waited past it ranks
    before small jobs submitted later: it finishes before the last of a stream of small jobs."""
    srv, ids = make_server(resident, pool_size=4096, schedule=pathtracer.SCHEDULE_DEADLINE, deadline_slowdown=1.0)
    try:
        big = ("spheres-small", 96, 96, 16, 10, True, 0)
        small = ("cornell-all", 32, 32, 4, 6, True, 0)
        j_big = submit(srv, ids, resident, big)
        smalls = []
        for _ in range(40):
            smalls.append(submit(srv, ids, resident, small))
            time.sleep(0.005)
        check_job(srv, j_big, frame_renderers, resident, big)
        for j in smalls:
            check_job(srv, j, frame_renderers, resident, small)
        assert srv.poll(j_big)["done_s"] < max(srv.poll(j)["done_s"] for j in smalls)
    finally:
        srv.close()


def test_tiny_pool_and_single_pass_ring(resident, frame_renderers):
    # 512 slots and one pass buffer per job: jobs wait on each other's slots and on their own folds
    srv, ids = make_server(resident, pool_size=512, ring_passes=1)
    try:
        jobs = JOBS[:4]
        jids = [submit(srv, ids, resident, job) for job in jobs]
        for jid, job in zip(jids, jobs):
            check_job(srv, jid, frame_renderers, resident, job)
    finally:
        srv.close()


def test_many_single_pixel_jobs(resident, frame_renderers):
    """1,200 jobs of one pixel in flight together: a regeneration block retires paths of more jobs and
    passes than its shared-memory pass table and plan-segment copy hold, so both fall back to
    global memory. Every image still equals the frame renderer's."""
    srv, ids = make_server(resident, pool_size=1 << 14, max_jobs=2048)
    try:
        jobs = [("cornell-all", 1 + (k % 2), 1, (1, 4)[k % 2], 3 + k % 3, True, 7 * k) for k in range(1200)]
        jids = [submit(srv, ids, resident, job) for job in jobs]
        for jid, job in zip(jids, jobs):
            check_job(srv, jid, frame_renderers, resident, job)
        assert srv.stats()["completed_jobs"] == len(jobs)
    finally:
        srv.close()


def test_one_job_at_a_time(resident, frame_renderers):
    srv, ids = make_server(resident, pool_size=1 << 16, max_active_jobs=1)
    try:
        jobs = JOBS[:3]
        jids = [submit(srv, ids, resident, job) for job in jobs]
        for jid, job in zip(jids, jobs):
            check_job(srv, jid, frame_renderers, resident, job)
        admits = [srv.poll(j)["admit_s"] for j in jids]
        dones = [srv.poll(j)["done_s"] for j in jids]
        # each job is admitted only after the previous one finished
        assert admits[1] >= dones[0] and admits[2] >= dones[1]
    finally:
        srv.close()


def test_budget_admission_and_refusal(resident, frame_renderers):
    name, w, h = "cornell-all", 64, 64
    # a budget for one such job at a time (about 0.61 MB: 64 B x 4096 in-flight paths, a ring of its 4
    # passes, accumulator and framebuffer; two jobs need 1.2 MB)
    budget = 700_000
    srv, ids = make_server(resident, pool_size=1 << 12, hbm_budget_bytes=budget)
    try:
        with pytest.raises(pathtracer.GptError) as e:
            srv.submit(ids[name], scenes.scene_camera(resident[name], 512, 512), 512, 512, 4, 4, True)
        assert e.value.code == 6
        job = (name, w, h, 4, 6, True, 0)
        jids = [submit(srv, ids, resident, job) for _ in range(3)]
        for jid in jids:
            check_job(srv, jid, frame_renderers, resident, job)
        st = srv.stats()
        assert st["admitted_high_water"] <= budget
        assert st["admitted_high_water"] == srv.poll(jids[0])["admitted_bytes"]
    finally:
        srv.close()


def test_cancel_running_and_queued(resident, frame_renderers):
    srv, ids = make_server(resident, pool_size=1 << 12, max_active_jobs=1)
    try:
        big = ("spheres-small", 256, 256, 64, 12, True, 0)
        small = ("cornell-all", 40, 30, 4, 6, True, 0)
        j_big = submit(srv, ids, resident, big)
        j_queued = submit(srv, ids, resident, small)
        srv.cancel(j_queued)
        srv.cancel(j_big)
        st = srv.wait(j_big, 300)
        assert st["state"] == "cancelled"
        assert srv.poll(j_queued)["state"] == "cancelled"
        # the server keeps working after cancellations
        j_ok = submit(srv, ids, resident, small)
        check_job(srv, j_ok, frame_renderers, resident, small)
    finally:
        srv.close()


def test_nee_without_emitters_matches_oracle(resident, frame_renderers, gpu_renderer):
    """No emitters with NEE on: the deterministic build equals the oracle bit for bit; the product
    build (CUDA's transcendentals) agrees per path within 1e-4."""
    import oracle
    s = resident["cornell-dark"]
    cam = scenes.scene_camera(s, 24, 24)
    o = oracle.OracleScene(s).render(cam, 24, 24, 4, 6, True)
    gpu_renderer.upload_scene(s)
    gpu_renderer.render_frame(cam, 24, 24, 4, 6, True)
    assert np.array_equal(gpu_renderer.sample_radiance().view(np.uint32), o["sample_radiance"].view(np.uint32))
    assert np.array_equal(gpu_renderer.framebuffer().reshape(-1), o["framebuffer"])
    r = frame_renderers["cornell-dark"]
    r.render_frame(cam, 24, 24, 4, 6, True)
    a, b = r.sample_radiance().astype(np.float64), o["sample_radiance"].astype(np.float64)
    assert np.all(np.abs(a - b) <= 1e-4 * np.maximum(np.abs(b), 1e-6))
    assert b.max() > 0


def test_batched_mix_sample_matches_frames(scene_factory):
    """A scaled-down sample of the 64-job batched mix (its scenes, seeded cameras, spp and depths,
    resolutions divided by 8) rendered together through the server: every image equals the frame
    renderer's for the same job, bit for bit."""
    import workloads
    names = ("spheres-10k", "spheres-200k")
    jobs = [j for j in workloads.batched_jobs() if j.scene in names][:8]
    assert len(jobs) >= 4
    resident = {n: scene_factory(n) for n in names}
    srv = pathtracer.Server(0, pool_size=1 << 18, hbm_budget_bytes=BUDGET)
    renderers = {}
    try:
        ids = {n: srv.add_scene(s) for n, s in resident.items()}
        small = []
        for j in jobs:
            w, h = max(8, j.width // 8), max(8, j.height // 8)
            cam = workloads.orbit_camera(np.random.default_rng(len(small)), w, h)
            small.append((j.scene, w, h, j.spp, j.depth, cam))
        jids = [srv.submit(ids[n], cam, w, h, spp, depth, True, keep_accumulation=True) for n, w, h, spp, depth, cam in small]
        for n in names:
            renderers[n] = pathtracer.Renderer(0)
            renderers[n].upload_scene(resident[n])
        for jid, (n, w, h, spp, depth, cam) in zip(jids, small):
            st = srv.wait(jid, 300)
            assert st["state"] == "done", srv.last_error()
            fb, acc = srv.result(jid, accumulation=True)
            r = renderers[n]
            r.render_frame(cam, w, h, spp, depth, True)
            assert np.array_equal(acc.view(np.uint32), r.accumulation().reshape(-1, 4).view(np.uint32)), (n, w, h, spp)
            assert np.array_equal(fb, r.framebuffer().reshape(-1))
    finally:
        srv.close()
        for r in renderers.values():
            r.close()
