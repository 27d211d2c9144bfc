// spk_tune.cu -- the schedule autotuner (include/spooky_b200.h, spk_autotune,
// spk_ensemble_autotune).  Included at the end of spk_api.cu (one
// translation unit).
//
// Each knob is a launch choice that leaves the arithmetic unchanged, so that
// a tuned context computes the same values as an untuned one:
//   tune_zl   lines per CTA of the z pass (shared memory per CTA against the
//             busy transform slots: the launcher's own choice is a model);
//   tune_nst  pipeline stages of the axis passes (TMA loads in flight against
//             CTAs per SM);
//   tune_rhs  CTAs per SM of the RHS grid (loads in flight against tail);
//   tune_kt   half-width tiles for the axis passes of axes up to 64 long
//             (fewer idle columns against fewer threads per CTA).
// Coordinate descent over the knobs, each candidate timed with CUDA events
// over whole recorded steps; the state and the step scalars are restored
// afterwards.

static float time_steps(spk_ctx* c, int steps, int* rc) {
    *rc = spk_advance(c, 1);   // records the step graph and warms it
    if (*rc) return 0.f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c->stream);
    *rc = spk_advance(c, steps);
    cudaEventRecord(e1, c->stream);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!*rc) *rc = launch_status(c);
    return ms / (float)std::max(steps, 1);
}

extern "C" int spk_autotune(spk_ctx* c, int steps, int* zl, int* nst, int* rhs, double* ms_before, double* ms_after) {
    if (!c || steps < 1) return SPK_ERR_ARG;
    if (c->p.heat_equation) return fail(c, SPK_ERR_UNSUPPORTED, "the heat-equation mode has no tunable passes");
    if (c->dirty) launch_clean(c);
    CK(cudaStreamSynchronize(c->stream));
    int rc = pull_scalars(c);
    if (rc) return rc;
    // save the state and the step scalars (restored at the end)
    const size_t sbytes = sizeof(double2) * c->nc * c->F * c->nb;
    void* saved = nullptr;
    if (cudaMalloc(&saved, sbytes) != cudaSuccess) return fail(c, SPK_ERR_ALLOC, "autotune: no room for a copy of the state");
    CK(cudaMemcpyAsync(saved, c->U, sbytes, cudaMemcpyDeviceToDevice, c->stream));
    std::vector<DevScalars> sc0(c->h_sc, c->h_sc + c->nb);
    const int h_step0 = c->h_step;

    drop_graphs(c);
    const float base = time_steps(c, steps, &rc);
    float best_ms = base;
    struct Knob { int* v; std::vector<int> cand; };
    // the tile width first: the stage count depends on it
    const bool short_axis = c->nx <= 64 || c->ny <= 64;
    Knob knobs[4] = {{&c->tune_kt, short_axis ? std::vector<int>{0, 2} : std::vector<int>{}},
                     {&c->tune_zl, {1, 2, 4, 8, 16, 32, 64}}, {&c->tune_nst, {1, 2, 3, 4}}, {&c->tune_rhs, {6, 12, 24, 48}}};
    for (int kq = 0; kq < 4 && !rc; kq++) {
        int best = *knobs[kq].v;
        for (int v : knobs[kq].cand) {
            *knobs[kq].v = v;
            drop_graphs(c);
            const float ms = time_steps(c, steps, &rc);
            if (rc) break;
            if (ms < best_ms) { best_ms = ms; best = v; }
        }
        *knobs[kq].v = best;
    }
    // restore the state and the step scalars; the next step records the tuned graph
    drop_graphs(c);
    cudaMemcpyAsync(c->U, saved, sbytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(c->sc, sc0.data(), sizeof(DevScalars) * c->nb, cudaMemcpyHostToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
    cudaFree(saved);
    c->h_step = h_step0;
    c->dirty = false;   // the saved state had been cleaned and scanned (its flag is restored too)
    if (rc) return rc;
    if (zl) *zl = c->tune_zl;
    if (nst) *nst = c->tune_nst;
    if (rhs) *rhs = c->tune_rhs;
    if (ms_before) *ms_before = base;
    if (ms_after) *ms_after = best_ms;
    return launch_status(c);
}

extern "C" int spk_get_schedule(const spk_ctx* c, int* zl, int* nst, int* rhs, int* tile_div) {
    if (!c) return SPK_ERR_ARG;
    if (zl) *zl = c->tune_zl;
    if (nst) *nst = c->tune_nst;
    if (rhs) *rhs = c->tune_rhs;
    if (tile_div) *tile_div = c->tune_kt == 2 ? 2 : 1;
    return SPK_OK;
}

extern "C" int spk_set_schedule(spk_ctx* c, int zl, int nst, int rhs, int tile_div) {
    if (!c) return SPK_ERR_ARG;
    if (zl < 0 || nst < 0 || nst > 4 || rhs < 0 || (tile_div != 0 && tile_div != 1 && tile_div != 2))
        return fail(c, SPK_ERR_ARG, "schedule: z_lines >= 0, axis_stages 0..4, rhs_ctas_per_sm >= 0, axis_tile_div 0, 1 or 2");
    CK(cudaStreamSynchronize(c->stream));
    c->tune_zl = zl;
    c->tune_nst = nst;
    c->tune_rhs = rhs;
    c->tune_kt = tile_div == 2 ? 2 : 0;
    drop_graphs(c);   // the next step records the new schedule
    return SPK_OK;
}

extern "C" int spk_ensemble_autotune(spk_ensemble* e, int steps) {
    if (!e || steps < 1) return SPK_ERR_ARG;
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return ens_fail("ensemble stream synchronisation failed", SPK_ERR_CUDA);
    for (size_t gq = 0; gq < e->group.size(); gq++) {
        spk_ctx* c = e->group[gq];
        if (c->p.heat_equation) continue;
        const int rc = spk_autotune(c, steps, nullptr, nullptr, nullptr, nullptr, nullptr);
        if (rc) return ens_fail("ensemble group " + std::to_string(gq) + ": " + c->err, rc);
    }
    if (e->have_graph) { cudaGraphExecDestroy(e->gexec); e->have_graph = false; }
    return SPK_OK;
}
