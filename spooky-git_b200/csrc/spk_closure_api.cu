// spk_closure_api.cu -- C ABI of the learned subgrid closure
// (include/spooky_b200.h, SPK_CLOSURE_*): weights into a context, spectral
// products, training samples from a fine-grid state, and the trainer.
// Included at the end of spk_api.cu (one translation unit).

extern "C" int spk_closure_nparam(int variant) {
    return (variant == 1 || variant == 2) ? (int)CL_NP : (variant == 3 ? (int)C3_NP : 0);
}

extern "C" int spk_closure_rows(int variant) {
    return (variant == 1 || variant == 2) ? SPK_CLOSURE_ROWS : (variant == 3 ? SPK_CLOSURE3_ROWS : 0);
}

extern "C" int spk_closure_set(spk_ctx* c, const float* params) {
    if (!c) return SPK_ERR_ARG;
    if (!c->p.closure) return fail(c, SPK_ERR_UNSUPPORTED, "the context was created without params.closure");
    if (params) {
        CK(cudaMemcpyAsync(c->d_cparams, params, sizeof(float) * (size_t)spk_closure_nparam(c->p.closure),
                           cudaMemcpyHostToDevice, c->stream));
        if (c->p.closure == 3) {
            c->launches++;
            k_closure3_pack<<<32, 256, 0, c->stream>>>(c->d_cparams, c->d_cimg);
            CK(cudaGetLastError());
        }
        CK(cudaStreamSynchronize(c->stream));
    }
    const bool on = params != nullptr;
    if (on != c->closure_on) {
        // the step graphs hold the pass layout: record them again
        drop_graphs(c);
        c->closure_on = on;
    }
    return SPK_OK;
}

extern "C" int spk_products(spk_ctx* c, const double* U, double* P, int* nprod) {
    if (!c || !U || !P) return SPK_ERR_ARG;
    if (!c->p.incompressible || c->p.boussinesq || c->nb != 1)
        return fail(c, SPK_ERR_UNSUPPORTED, "spk_products covers single HD and MHD contexts");
    const int np = c->p.mhd ? 8 : 5;
    c->user_U = U;
    pass_x_inverse(c, (const double2*)U, true);
    c->user_U = nullptr;
    pass_y_inverse(c, true);
    pass_z_products(c, false);
    pass_y_forward(c, c->nout, c->bufA, c->bufB);
    pass_x_forward(c);
    const void* nl = chan(c, c->bufA, c->out_T);
    const int grid = ew_blocks(c->nc * np);
    c->launches++;
    if (c->fp32) k_products_out<float><<<grid, 256, 0, c->stream>>>(c->g, (const C2<float>*)nl, np, (double2*)P);
    else k_products_out<double><<<grid, 256, 0, c->stream>>>(c->g, (const C2<double>*)nl, np, (double2*)P);
    if (nprod) *nprod = np;
    return launch_status(c);
}

// Real fields R[nch][nr] (FP64) of nch spectral channels X[nch][Nc] in the
// state layout: x and y inverse passes and the z to-real pass, F channels at
// a time.  X must hold a multiple of F channels (the tensor map of each
// chunk spans F channels; only the chunk's own are read).
static int c2r_channels(spk_ctx* c, const double2* X, int nch, double* R) {
    for (int c0 = 0; c0 < nch; c0 += c->F) {
        const int m = std::min(c->F, nch - c0);
        c->user_U = X + (size_t)c0 * c->nc;
        AxisArgs a = axis_args(c, 0);
        a.scale = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
        add_job(c, a, c->user_U, c->bufA, m, 1, 0, 0);
        axis(c, a, +1);
        c->user_U = nullptr;
        AxisArgs b = axis_args(c, 1);
        add_job(c, b, c->bufA, c->bufB, m, 0, 0, 0);
        axis(c, b, +1);
        ZArgs z = z_args(c);
        z.mode = ZM_TO_REAL;
        z.nin = m;
        z.real_out = R + (size_t)c0 * c->nr;
        zpass(c, z);
        if (c->sticky) break;
    }
    return launch_status(c);
}

static size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }
static int pad_to(int n, int F) { return ((n + F - 1) / F) * F; }

struct SampleScratch { size_t pf, pt, pc, gs, rt, rg, rgf, total; };
static SampleScratch sample_scratch(const spk_ctx* f, const spk_ctx* c) {
    const int np = c->p.mhd ? 8 : 5;
    SampleScratch s;
    s.pf = 0;
    s.pt = s.pf + al256(sizeof(double2) * f->nc * np);
    s.pc = s.pt + al256(sizeof(double2) * c->nc * pad_to(np, c->F));
    s.gs = s.pc + al256(sizeof(double2) * c->nc * np);
    s.rt = s.gs + al256(sizeof(double2) * c->nc * pad_to(18, c->F));
    s.rg = s.rt + al256(sizeof(double) * c->nr * np);
    s.rgf = s.rg + al256(sizeof(double) * c->nr * 18);
    // the whole field's gradients, apart from the model's input in variant 2
    s.total = s.rgf + (c->p.closure == 2 ? al256(sizeof(double) * c->nr * 18) : 0);
    return s;
}

static const char* samples_mismatch(const spk_ctx* f, const spk_ctx* c) {
    if (!f->p.incompressible || !c->p.incompressible || f->p.boussinesq || c->p.boussinesq)
        return "closure samples need HD or MHD contexts";
    if (f->p.mhd != c->p.mhd) return "the fine and coarse contexts differ in their modules";
    if (f->nb != 1 || c->nb != 1) return "closure samples need single-box contexts";
    if (f->p.lx != c->p.lx || f->p.ly != c->p.ly || f->p.lz != c->p.lz) return "the contexts have different boxes";
    if (c->nx > f->nx || c->ny > f->ny || c->nz > f->nz) return "the coarse grid is finer than the fine grid";
    return nullptr;
}

extern "C" int spk_closure_samples_size(const spk_ctx* f, const spk_ctx* c, size_t* bytes, size_t* ns) {
    if (!f || !c) return fail(nullptr, SPK_ERR_ARG, "null context");
    if (const char* why = samples_mismatch(f, c)) return fail(nullptr, SPK_ERR_UNSUPPORTED, why);
    if (bytes) *bytes = sample_scratch(f, c).total;
    if (ns) *ns = c->nr;
    return SPK_OK;
}

extern "C" int spk_closure_samples(spk_ctx* f, const double* Uf, spk_ctx* c, float* X, size_t stride, void* scratch,
                                   size_t scratch_bytes) {
    if (!f || !c || !Uf || !X || !scratch) return SPK_ERR_ARG;
    if (const char* why = samples_mismatch(f, c)) return fail(c, SPK_ERR_UNSUPPORTED, why);
    const SampleScratch sl = sample_scratch(f, c);
    if (scratch_bytes < sl.total) return fail(c, SPK_ERR_ARG, "scratch smaller than spk_closure_samples_size");
    if (stride < c->nr) return fail(c, SPK_ERR_ARG, "sample row stride below the coarse point count");
    char* base = (char*)scratch;
    double2* Pf = (double2*)(base + sl.pf);
    double2* Pt = (double2*)(base + sl.pt);
    double2* Pc = (double2*)(base + sl.pc);
    double2* Gs = (double2*)(base + sl.gs);
    double* Rt = (double*)(base + sl.rt);
    double* Rg = (double*)(base + sl.rg);
    double* Rgf = c->p.closure == 2 ? (double*)(base + sl.rgf) : nullptr;
    const int np = c->p.mhd ? 8 : 5;
    // products of the fine state (without the closure)
    const bool fon = f->closure_on;
    f->closure_on = false;
    int rc = spk_products(f, Uf, (double*)Pf, nullptr);
    f->closure_on = fon;
    if (rc) return fail(c, rc, f->err);
    CK(cudaStreamSynchronize(f->stream));
    // the filtered state into the coarse context; the filtered products
    TruncArgs t;
    t.fnx = f->nx; t.fny = f->ny; t.fnzh = f->nzh;
    t.cnx = c->nx; t.cny = c->ny; t.cnzh = c->nzh;
    t.mx = c->g.mx; t.my = c->g.my; t.mz = c->g.mz;
    t.scale = (double)c->nr / (double)f->nr;
    t.src = (const double2*)Uf; t.dst = c->U; t.nch = c->F;
    k_truncate<<<ew_blocks(c->nc * c->F), 256, 0, c->stream>>>(t);
    t.src = Pf; t.dst = Pt; t.nch = np;
    k_truncate<<<ew_blocks(c->nc * np), 256, 0, c->stream>>>(t);
    c->launches += 2;
    c->dirty = true;
    // products of the filtered state on the coarse grid (without the closure)
    const bool con = c->closure_on;
    c->closure_on = false;
    rc = spk_products(c, (const double*)c->U, (double*)Pc, nullptr);
    c->closure_on = con;
    if (rc) return rc;
    k_sub<<<ew_blocks(c->nc * np), 256, 0, c->stream>>>(Pt, Pc, c->nc * np);
    c->launches++;
    rc = c2r_channels(c, Pt, np, Rt);
    if (rc) return rc;
    // gradients of the filtered state: the whole field's (variant 2: and those
    // of its small scales, the model's input)
    for (int pass = 0; pass < (Rgf ? 2 : 1); pass++) {
        const bool hp = Rgf && pass == 1;
        CK(cudaMemsetAsync(Gs, 0, sizeof(double2) * c->nc * 18, c->stream));
        k_gradients<<<ew_blocks(c->nc), 256, 0, c->stream>>>(c->g, c->U, c->VEL, c->MAG, c->p.mhd ? 2 : 1,
                                                              hp ? c->hp_k2 : 0.0, Gs);
        c->launches++;
        rc = c2r_channels(c, Gs, 18, Rgf && !hp ? Rgf : Rg);
        if (rc) return rc;
    }
    k_closure_rows<<<ew_blocks(c->nr), 256, 0, c->stream>>>(Rg, Rgf, Rt, np, c->nr, c->delta2, X, stride,
                                                             c->p.closure == 3 ? 1 : 0);
    c->launches++;
    return launch_status(c);
}

// ---------------------------------------------------------------------------
// shell spectra (diagnostics)
// ---------------------------------------------------------------------------
extern "C" int spk_spectrum(spk_ctx* c, int f1, int f2, double* out, int max_bins, int* nbins, double* deltak,
                            double* total) {
    if (!c || f1 < 0 || f2 < 0 || f1 >= c->F || f2 >= c->F) return SPK_ERR_ARG;
    if (nbins) *nbins = c->nbins;
    if (deltak) *deltak = c->deltak;
    if (c->nbins < 1) return fail(c, SPK_ERR_UNSUPPORTED, "no spectral bins for this grid");
    CK(cudaMemsetAsync(c->d_spec, 0, sizeof(double) * (size_t)(c->nbins + 1), c->stream));
    const double inv_n = 1.0 / ((double)c->nx * (double)c->ny * (double)c->nz);
    const int grid = (int)std::min<size_t>((c->nc + 255) / 256, (size_t)c->num_sms * 8);
    k_spectrum<<<grid, 256, sizeof(double) * (size_t)c->nbins, c->stream>>>(
        c->g, c->U + (size_t)f1 * c->nc, c->U + (size_t)f2 * c->nc, c->nbins, c->deltak, inv_n, c->d_spec);
    c->launches++;
    int rc = launch_status(c);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->h_sums, c->d_spec + c->nbins, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    std::vector<double> h((size_t)c->nbins);
    CK(cudaMemcpyAsync(h.data(), c->d_spec, sizeof(double) * (size_t)c->nbins, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (out) for (int m = 0; m < std::min(max_bins, c->nbins); m++) out[m] = h[(size_t)m];
    if (total) *total = c->h_sums[0];
    return SPK_OK;
}

// ---------------------------------------------------------------------------
// trainer
// ---------------------------------------------------------------------------
#define SPK_TRAIN_HIST 65536

struct spk_trainer {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int variant = 1;                 // 1 (also 2): the eddy-coefficient network; 3: the tensor network
    int np = CL_NP;                  // parameters
    unsigned char* img = nullptr;    // variant 3: the packed BF16 image of params
    float *params = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *partial = nullptr;
    float *hist = nullptr, *h_hist = nullptr;
    const float* X = nullptr;
    size_t n = 0, stride = 0;
    float w0 = 1.f, w1 = 1.f, w2 = 0.f;
    int t = 0;                       // Adam steps taken
    unsigned long long cursor = 0;   // samples drawn so far
};

static size_t grad_smem() { return sizeof(float) * (((CL_NP + 3) & ~3) + (size_t)CL_ROWS * CL_LDS); }

#define TCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return fail(nullptr, SPK_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

extern "C" int spk_trainer_create(void* stream, spk_trainer** out) { return spk_trainer_create_variant(stream, 1, out); }

static int train_blocks(const spk_trainer* tr) { return tr->variant == 3 ? 148 : CL_MAXBLK; }

extern "C" int spk_trainer_create_variant(void* stream, int variant, spk_trainer** out) {
    if (!out) return fail(nullptr, SPK_ERR_ARG, "null argument");
    *out = nullptr;
    if (spk_closure_nparam(variant) == 0) return fail(nullptr, SPK_ERR_ARG, "closure variant must be 1, 2 or 3");
    spk_trainer* tr = new spk_trainer();
    tr->variant = variant == 3 ? 3 : 1;
    tr->np = spk_closure_nparam(variant);
    auto bail = [&](int rc) { spk_trainer_destroy(tr); return rc; };
    if (stream) tr->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&tr->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(nullptr, SPK_ERR_CUDA, "stream creation failed"));
        tr->own_stream = true;
    }
    const size_t np = (size_t)tr->np;
    if (cudaMalloc(&tr->params, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&tr->m, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&tr->v, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&tr->grad, sizeof(float) * np) != cudaSuccess ||
        cudaMalloc(&tr->partial, sizeof(float) * (size_t)train_blocks(tr) * (np + 1)) != cudaSuccess ||
        cudaMalloc(&tr->hist, sizeof(float) * SPK_TRAIN_HIST) != cudaSuccess ||
        cudaMallocHost(&tr->h_hist, sizeof(float) * SPK_TRAIN_HIST) != cudaSuccess ||
        (tr->variant == 3 && cudaMalloc(&tr->img, (size_t)C3_ALL_BYTES) != cudaSuccess))
        return bail(fail(nullptr, SPK_ERR_ALLOC, "trainer allocation failed"));
    cudaMemset(tr->params, 0, sizeof(float) * np);
    cudaMemset(tr->m, 0, sizeof(float) * np);
    cudaMemset(tr->v, 0, sizeof(float) * np);
    if (cudaFuncSetAttribute(k_closure_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem()) != cudaSuccess ||
        cudaFuncSetAttribute(k_closure3_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C3G_BYTES) != cudaSuccess)
        return bail(fail(nullptr, SPK_ERR_CUDA, "shared-memory opt-in of the gradient kernel failed"));
    *out = tr;
    return SPK_OK;
}

extern "C" int spk_trainer_destroy(spk_trainer* tr) {
    if (!tr) return SPK_OK;
    cudaFree(tr->params); cudaFree(tr->m); cudaFree(tr->v); cudaFree(tr->grad); cudaFree(tr->partial);
    cudaFree(tr->hist);
    cudaFree(tr->img);
    if (tr->h_hist) cudaFreeHost(tr->h_hist);
    if (tr->own_stream) cudaStreamDestroy(tr->stream);
    delete tr;
    return SPK_OK;
}

extern "C" int spk_trainer_set_params(spk_trainer* tr, const float* params) {
    if (!tr || !params) return fail(nullptr, SPK_ERR_ARG, "null argument");
    TCK(cudaMemcpyAsync(tr->params, params, sizeof(float) * tr->np, cudaMemcpyHostToDevice, tr->stream));
    TCK(cudaMemsetAsync(tr->m, 0, sizeof(float) * tr->np, tr->stream));
    TCK(cudaMemsetAsync(tr->v, 0, sizeof(float) * tr->np, tr->stream));
    TCK(cudaStreamSynchronize(tr->stream));
    tr->t = 0;
    return SPK_OK;
}

extern "C" int spk_trainer_get_params(spk_trainer* tr, float* params) {
    if (!tr || !params) return fail(nullptr, SPK_ERR_ARG, "null argument");
    TCK(cudaMemcpyAsync(params, tr->params, sizeof(float) * tr->np, cudaMemcpyDeviceToHost, tr->stream));
    TCK(cudaStreamSynchronize(tr->stream));
    return SPK_OK;
}

extern "C" int spk_trainer_set_samples(spk_trainer* tr, const float* X, size_t n, size_t stride, const float w[3]) {
    if (!tr || !X || n == 0 || stride < n || !w) return fail(nullptr, SPK_ERR_ARG, "bad samples");
    tr->X = X; tr->n = n; tr->stride = stride; tr->w0 = w[0]; tr->w1 = w[1]; tr->w2 = w[2];
    tr->cursor = 0;
    return SPK_OK;
}

// one gradient evaluation over m samples (minibatch: drawn from the cursor)
static void trainer_grad(spk_trainer* tr, size_t m, bool minibatch, float* loss_out) {
    TrainArgs a;
    a.X = tr->X; a.n = tr->n; a.stride = tr->stride; a.m = m;
    a.minibatch = minibatch ? 1 : 0;
    // a multiplier coprime with n: consecutive draws walk the samples in a scattered order
    unsigned long long mult = tr->n > 2 ? ((unsigned long long)((double)tr->n * 0.6180339887498949) | 1ull) : 1ull;
    auto gcd = [](unsigned long long x, unsigned long long y) { while (y) { unsigned long long r = x % y; x = y; y = r; } return x; };
    while (tr->n > 2 && gcd(mult, tr->n) != 1) mult += 2;
    a.a = mult % (tr->n > 0 ? tr->n : 1);
    a.c = tr->n / 3;
    a.base = tr->cursor;
    a.params = tr->params; a.w0 = tr->w0; a.w1 = tr->w1; a.w2 = tr->w2;
    a.partial = tr->partial;
    if (tr->variant == 3) {
        // the tensor network: BF16 image of the FP32 masters, then chunks of 64 samples
        Train3Args b;
        b.X = a.X; b.n = a.n; b.stride = a.stride; b.m = a.m; b.minibatch = a.minibatch;
        b.a = a.a; b.c = a.c; b.base = a.base;
        b.img = tr->img; b.w0 = a.w0; b.w1 = a.w1; b.w2 = a.w2; b.partial = tr->partial;
        const int nblk = (int)std::min<size_t>((size_t)train_blocks(tr), (m + C3_CH - 1) / C3_CH);
        k_closure3_pack<<<32, 256, 0, tr->stream>>>(tr->params, tr->img);
        k_closure3_grad<<<nblk, 128, C3G_BYTES, tr->stream>>>(b);
        k_closure_reduce_n<<<(C3_NP + 1 + 127) / 128, 128, 0, tr->stream>>>(tr->partial, nblk, C3_NP, 1.0 / (double)m,
                                                                            tr->grad, loss_out);
        return;
    }
    const int nblk = (int)std::min<size_t>(CL_MAXBLK, (m + CL_CHUNK - 1) / CL_CHUNK);
    k_closure_grad<<<nblk, CL_CHUNK, grad_smem(), tr->stream>>>(a);
    k_closure_reduce<<<(CL_NP + 1 + 127) / 128, 128, 0, tr->stream>>>(tr->partial, nblk, 1.0 / (double)m, tr->grad,
                                                                        loss_out);
}

extern "C" int spk_trainer_loss_grad(spk_trainer* tr, float* loss, float* grad) {
    if (!tr || !tr->X) return fail(nullptr, SPK_ERR_ARG, "trainer without samples");
    trainer_grad(tr, tr->n, false, tr->hist);
    TCK(cudaGetLastError());
    if (grad) TCK(cudaMemcpyAsync(grad, tr->grad, sizeof(float) * tr->np, cudaMemcpyDeviceToHost, tr->stream));
    TCK(cudaMemcpyAsync(tr->h_hist, tr->hist, sizeof(float), cudaMemcpyDeviceToHost, tr->stream));
    TCK(cudaStreamSynchronize(tr->stream));
    if (loss) *loss = tr->h_hist[0];
    return SPK_OK;
}

extern "C" int spk_trainer_train(spk_trainer* tr, int nsteps, int batch, float lr, float* loss_hist) {
    if (!tr || !tr->X || nsteps < 0 || batch < 1) return fail(nullptr, SPK_ERR_ARG, "bad training request");
    for (int done = 0; done < nsteps;) {
        const int k = std::min(nsteps - done, SPK_TRAIN_HIST);
        for (int i = 0; i < k; i++) {
            trainer_grad(tr, (size_t)batch, true, tr->hist + i);
            tr->t++;
            tr->cursor += (unsigned long long)batch;
            if (tr->variant == 3)
                k_closure_adam_n<<<(C3_NP + 255) / 256, 256, 0, tr->stream>>>(tr->params, tr->grad, tr->m, tr->v, C3_NP,
                                                                              tr->t, lr);
            else
                k_closure_adam<<<(CL_NP + 255) / 256, 256, 0, tr->stream>>>(tr->params, tr->grad, tr->m, tr->v, tr->t, lr);
        }
        TCK(cudaGetLastError());
        if (loss_hist) {
            TCK(cudaMemcpyAsync(tr->h_hist, tr->hist, sizeof(float) * k, cudaMemcpyDeviceToHost, tr->stream));
            TCK(cudaStreamSynchronize(tr->stream));
            memcpy(loss_hist + done, tr->h_hist, sizeof(float) * k);
        }
        done += k;
    }
    TCK(cudaStreamSynchronize(tr->stream));
    return SPK_OK;
}
