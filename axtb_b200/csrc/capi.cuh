// C ABI (include/axtb_gpu.h, include/axtb_gpu_debug.h) over the batch engine.
#pragma once

// total energies of the batch on the device: fixed (repulsion + ATM) + electronic
namespace axg {
__global__ void k_total_energy(int nmol, const double* erep, const double* eatm, const double* eel, double* out) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < nmol) out[m] = erep[m] + eatm[m] + eel[m];
}
}  // namespace axg

static int status_code(int bits, int conv) {
    if (bits & (axg::ST_HISTORY)) return AXTB_ERR_SCF_NOT_CONVERGED;
    if (bits != 0) return AXTB_ERR_NUMERICAL;
    if (!conv) return AXTB_ERR_SCF_NOT_CONVERGED;
    return AXTB_OK;
}

void AxtbBatch::extract(AxtbResult* outs, int32_t* status, bool want_grad) {
    vector<double> eel(nmol), erep(nmol), eatm(nmol), terms((size_t)nmol * 8), de(nmol), res(nmol);
    vector<int> st_(nmol), conv(nmol), nit(nmol), nit0(nmol), used(nmol);
    vector<double> esolv(nmol, 0.0);
    if (B.solv) CK(cudaMemcpyAsync(esolv.data(), S.sv_emol, sizeof(double) * nmol, cudaMemcpyDeviceToHost, st));
    vector<double> grad((size_t)natT * 3), qat(natT), dp((size_t)natT * 3), qp((size_t)natT * 6), qsh(nshT);
    CK(cudaMemcpyAsync(eel.data(), S.energy, sizeof(double) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(erep.data(), S.e_fixed, sizeof(double) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(eatm.data(), d_eatm, sizeof(double) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(terms.data(), S.terms, sizeof(double) * nmol * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(de.data(), S.de, sizeof(double) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(res.data(), S.res, sizeof(double) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(st_.data(), S.status, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(conv.data(), S.conv, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nit.data(), S.niter, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(nit0.data(), S.niter_prev, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(used.data(), S.mix_used, sizeof(int) * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(qat.data(), S.qat_out, sizeof(double) * natT, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(dp.data(), S.dp_out, sizeof(double) * natT * 3, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(qp.data(), S.qp_out, sizeof(double) * natT * 6, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(qsh.data(), S.qsh_out, sizeof(double) * nshT, cudaMemcpyDeviceToHost, st));
    if (want_grad) CK(cudaMemcpyAsync(grad.data(), S.grad, sizeof(double) * natT * 3, cudaMemcpyDeviceToHost, st));
    // the electronic structure, when a result asks for it
    bool levels = std::any_of(outs, outs + nmol, [](const AxtbResult& r) { return r.emo || r.focc || r.focc_alpha; });
    vector<double> emo, focc, focca, ef(2 * (size_t)nmol);
    if (levels) {
        emo.resize(naoT);
        focc.resize(naoT);
        focca.resize(naoT);
        CK(cudaMemcpyAsync(emo.data(), S.emo, sizeof(double) * naoT, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(focc.data(), S.focc, sizeof(double) * naoT, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(focca.data(), S.focc_a, sizeof(double) * naoT, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaMemcpyAsync(ef.data(), S.efermi, sizeof(double) * 2 * nmol, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    d2h_bytes += (long long)(sizeof(double) * (nmol * (B.solv ? 17 : 16) + (size_t)natT * 10 + nshT) +
                             sizeof(int) * nmol * 5) +
                 (want_grad ? (long long)sizeof(double) * natT * 3 : 0) +
                 (levels ? (long long)sizeof(double) * naoT * 3 : 0);
    // phase times of this pass (events recorded by run on the stream)
    float ms[3] = {0.0f, 0.0f, 0.0f}, tot = 0.0f;
    for (int k = 0; k < 3; k++) CK(cudaEventElapsedTime(&ms[k], phase_ev[k], phase_ev[k + 1]));
    CK(cudaEventElapsedTime(&tot, phase_ev[0], phase_ev[3]));
    for (int m = 0; m < nmol; m++) {
        AxtbResult& r = outs[m];
        int a0 = m_at0[m], nat = mols[m].nat;
        r.energy = erep[m] + eatm[m] + eel[m];
        for (int k = 0; k < 8; k++) r.terms[k] = terms[(size_t)m * 8 + k];
        r.terms[0] = erep[m];
        r.terms[1] += eatm[m];
        // iterations of the converged attempt; of both attempts when none converged
        // (crates/axtb/src/xtb.rs:624-645)
        r.iterations = conv[m] ? nit[m] : nit[m] + nit0[m];
        r.converged = conv[m];
        r.mixer_used = used[m];
        r.solvation = esolv[m];
        r.energy_change = de[m];
        r.residual = res[m];
        r.status = status_code(st_[m], conv[m]);
        if (status) status[m] = r.status;
        r.nao = mols[m].nao;
        r.fermi_levels[0] = ef[2 * (size_t)m];
        r.fermi_levels[1] = ef[2 * (size_t)m + 1];
        r.electronic_temperature = B.kt > 0.0 ? opt.etemp : 0.0;
        r.warm_start = m < (int)h_warm.size() ? h_warm[m] : 0;
        r.fallback_iterations = used[m] == 2 ? nit0[m] : 0;
        for (int k = 0; k < 3; k++) r.timings[k] = ms[k] * 1e-3;
        r.timings[3] = tot * 1e-3;
        if (levels) {
            size_t o0 = m_ao0[m], n = mols[m].nao;
            if (r.emo) std::memcpy(r.emo, emo.data() + o0, sizeof(double) * n);
            if (r.focc) std::memcpy(r.focc, focc.data() + o0, sizeof(double) * n);
            if (r.focc_alpha) std::memcpy(r.focc_alpha, focca.data() + o0, sizeof(double) * n);
        }
        if (want_grad && r.gradient)
            std::memcpy(r.gradient, grad.data() + (size_t)a0 * 3, sizeof(double) * nat * 3);
        if (r.charges) std::memcpy(r.charges, qat.data() + a0, sizeof(double) * nat);
        if (r.dpat) std::memcpy(r.dpat, dp.data() + (size_t)a0 * 3, sizeof(double) * nat * 3);
        if (r.qpat) std::memcpy(r.qpat, qp.data() + (size_t)a0 * 6, sizeof(double) * nat * 6);
        if (r.qsh) std::memcpy(r.qsh, qsh.data() + m_sh0[m], sizeof(double) * mols[m].nsh);
        if (r.dipole) {
            for (int k = 0; k < 3; k++) {
                double s = 0.0;
                for (int i = 0; i < nat; i++) s += qat[a0 + i] * mols[m].xyz[3 * i + k] + dp[(size_t)(a0 + i) * 3 + k];
                r.dipole[k] = s;
            }
        }
    }
}

// A molecule's SCC moments (ScfGuess, crates/axtb/src/xtb.rs:204-215): shell charges (nsh),
// atomic dipoles (nat*3) and atomic quadrupoles (nat*6).
struct Moments {
    vector<double> qsh, dp, qp;
};

// the moments of molecule m into the device buffers a warm start reads (the output moments of
// the previous run; atomic charges summed from the shells)
void AxtbBatch::put_moments(int m, const Moments& w) {
    int a0 = m_at0[m], s0 = m_sh0[m], nat = mols[m].nat;
    vector<double> qat(nat, 0.0);
    for (int i = 0, s = 0; i < nat; i++)
        for (int k = 0; k < gfn2tab::NSHELL[mols[m].Z[i] - 1]; k++, s++) qat[i] += w.qsh[s];
    CK(cudaMemcpyAsync(S.qsh_out + s0, w.qsh.data(), sizeof(double) * w.qsh.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.qat_out + a0, qat.data(), sizeof(double) * nat, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.dp_out + 3LL * a0, w.dp.data(), sizeof(double) * 3 * nat, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.qp_out + 6LL * a0, w.qp.data(), sizeof(double) * 6 * nat, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
}

// the output moments of molecule m in the last run
Moments AxtbBatch::get_moments(int m) {
    Moments w;
    int a0 = m_at0[m], s0 = m_sh0[m], nat = mols[m].nat;
    w.qsh.resize(mols[m].nsh);
    w.dp.resize(3 * (size_t)nat);
    w.qp.resize(6 * (size_t)nat);
    CK(cudaMemcpyAsync(w.qsh.data(), S.qsh_out + s0, sizeof(double) * w.qsh.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(w.dp.data(), S.dp_out + 3LL * a0, sizeof(double) * 3 * nat, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(w.qp.data(), S.qp_out + 6LL * a0, sizeof(double) * 6 * nat, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return w;
}

static Moments moments_from(const HostMol& m, const double* qsh, const double* dpat, const double* qpat) {
    if (!qsh || !dpat || !qpat) throw Fail(AXTB_ERR_INPUT, "moments: shell charges, dipoles and quadrupoles are all needed");
    Moments w;
    w.qsh.assign(qsh, qsh + m.nsh);
    w.dp.assign(dpat, dpat + 3 * (size_t)m.nat);
    w.qp.assign(qpat, qpat + 6 * (size_t)m.nat);
    for (const auto* v : {&w.qsh, &w.dp, &w.qp})
        for (double x : *v)
            if (!std::isfinite(x)) throw Fail(AXTB_ERR_INPUT, "moments: non-finite value");
    return w;
}

static void moments_to(const Moments& w, double* qsh, double* dpat, double* qpat) {
    if (qsh) std::memcpy(qsh, w.qsh.data(), sizeof(double) * w.qsh.size());
    if (dpat) std::memcpy(dpat, w.dp.data(), sizeof(double) * w.dp.size());
    if (qpat) std::memcpy(qpat, w.qp.data(), sizeof(double) * w.qp.size());
}

// The calculator of one molecule (axtb::Calculator): its options, the molecule, the device
// batch (made at the first single point) and the moments the next SCF starts from (`start`,
// crates/axtb/src/calculator.rs:185-206; `given` when they were set from outside).
struct AxtbHandle {
    HostMol mol;
    Opt opt;
    AxtbBatch* batch = nullptr;
    bool have_start = false, given = false;
    Moments start;
    std::string err;
    ~AxtbHandle() { delete batch; }
};

static Opt to_opt(const AxtbOptions* o) {
    Opt r;
    if (o) {
        r.acc = o->accuracy;
        r.etemp = o->etemp;
        r.max_iter = o->max_iter;
        r.damping = o->damping;
        r.guess = o->guess;
        r.precision = o->precision;
        r.device = o->device;
        r.mixer = o->mixer;
        r.conventions = o->conventions;
        r.solv = o->solvation;
        r.solvent = o->solvent ? o->solvent : "";
        r.solv_state = o->solvation_state;
        r.dispersion = o->dispersion != 0 ? 1 : 0;
        r.band_max_nao = o->band_max_nao;
        r.grid_min_nao = o->grid_min_nao;
    }
    return r;
}

static HostMol to_mol(const AxtbMol& m) {
    HostMol h;
    if (m.nat <= 0 || !m.numbers || !m.positions) throw Fail(AXTB_ERR_INPUT, "molecule has no atoms");
    h.nat = m.nat;
    h.Z.assign(m.numbers, m.numbers + m.nat);
    h.xyz.assign(m.positions, m.positions + 3 * (size_t)m.nat);
    h.charge = m.charge;
    h.uhf = m.uhf;
    check_molecule(h);
    return h;
}

template <class F>
static int guarded(std::string* sink, F&& f) {
    try {
        f();
        return AXTB_OK;
    } catch (const Fail& e) {
        g_last_error = e.what();
        if (sink) *sink = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        if (sink) *sink = e.what();
        return AXTB_ERR_DEVICE;
    }
}

extern "C" {

void axtb_gpu_default_options(AxtbOptions* o) {
    if (!o) return;
    o->accuracy = 1.0;
    o->etemp = 300.0;
    o->max_iter = 250;
    o->damping = 0.4;
    o->guess = 0;
    o->precision = 0;
    o->device = 0;
    o->mixer = -1;
    o->conventions = 0;
    o->solvation = -1;
    o->solvent = nullptr;
    o->solvation_state = 0;
    o->dispersion = 1;
    o->band_max_nao = -1;
    o->grid_min_nao = -1;
}

int axtb_gpu_basis_size(const int32_t* numbers, int32_t nat, int32_t* nsh, int32_t* nao) {
    int s = 0, a = 0;
    for (int i = 0; i < nat; i++) {
        int z = numbers[i];
        if (z < 1 || z > 86) return AXTB_ERR_UNSUPPORTED_ELEMENT;
        for (int k = 0; k < gfn2tab::NSHELL[z - 1]; k++) {
            s++;
            a += 2 * gfn2tab::ANG_SHELL[z - 1][k] + 1;
        }
    }
    if (nsh) *nsh = s;
    if (nao) *nao = a;
    return AXTB_OK;
}

int axtb_gpu_create(const int32_t* numbers, int32_t nat, double charge, int32_t uhf, const AxtbOptions* opts,
                    AxtbHandle** out) {
    if (!out) return AXTB_ERR_INPUT;
    *out = nullptr;
    AxtbHandle* h = new AxtbHandle();
    int rc = guarded(nullptr, [&] {
        h->opt = to_opt(opts);
        check_options(h->opt);
        if (nat <= 0 || !numbers) throw Fail(AXTB_ERR_INPUT, "molecule has no atoms");
        h->mol.nat = nat;
        h->mol.Z.assign(numbers, numbers + nat);
        h->mol.xyz.assign(3 * (size_t)nat, 0.0);
        for (int i = 0; i < nat; i++) h->mol.xyz[3 * i] = 10.0 * i;  // placeholder positions, replaced per call
        h->mol.charge = charge;
        h->mol.uhf = uhf;
        check_molecule(h->mol);
    });
    if (rc != AXTB_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return AXTB_OK;
}

int axtb_gpu_singlepoint(AxtbHandle* h, const double* positions, int32_t want_gradient, AxtbResult* out) {
    if (!h || !positions || !out) return AXTB_ERR_INPUT;
    return guarded(&h->err, [&] {
        HostMol m = h->mol;
        m.xyz.assign(positions, positions + 3 * (size_t)m.nat);
        check_molecule(m);
        if (!h->batch) {
            h->batch = new AxtbBatch();
            h->batch->build({m}, h->opt);
        }
        AxtbBatch& b = *h->batch;
        b.mols[0].xyz = m.xyz;
        b.upload_positions(m.xyz.data(), false);
        int32_t st = 0;
        // warm start from the previous geometry's (or the given) moments, then once more from
        // the guess when that did not converge (crates/axtb/src/calculator.rs:194-206; the
        // ladder climbs on ScfNotConverged only, crates/base/src/method/retry.rs:119-158)
        bool warm = h->have_start;
        bool lv = out->emo || out->focc || out->focc_alpha;
        if (warm) b.put_moments(0, h->start);
        h->have_start = h->given = false;
        b.run(want_gradient != 0, warm, lv);
        b.extract(out, &st, want_gradient != 0);
        if (st == AXTB_ERR_SCF_NOT_CONVERGED && warm) {
            b.run(want_gradient != 0, false, lv);
            b.extract(out, &st, want_gradient != 0);
        }
        if (st == AXTB_OK) {
            h->start = b.get_moments(0);
            h->have_start = true;
        }
        if (st != AXTB_OK) {
            char msg[160];
            std::snprintf(msg, sizeof msg, "SCF failed: status %d after %d iterations (dE %.3e, residual %.3e)", st,
                          out->iterations, out->energy_change, out->residual);
            throw Fail(st, msg);
        }
    });
}

void axtb_gpu_destroy(AxtbHandle* h) { delete h; }

int axtb_gpu_last_error(const AxtbHandle* h, char* buf, size_t len) {
    const std::string& s = h ? h->err : g_last_error;
    if (buf && len > 0) {
        size_t n = std::min(len - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return (int)s.size();
}

int axtb_gpu_get_moments(const AxtbHandle* h, double* qsh, double* dpat, double* qpat) {
    if (!h) return AXTB_ERR_INPUT;
    if (!h->have_start) {
        g_last_error = "the calculator has no moments (no converged single point and none given)";
        return AXTB_ERR_INPUT;
    }
    moments_to(h->start, qsh, dpat, qpat);
    return AXTB_OK;
}

int axtb_gpu_set_moments(AxtbHandle* h, const double* qsh, const double* dpat, const double* qpat, int32_t given) {
    if (!h) return AXTB_ERR_INPUT;
    return guarded(&h->err, [&] {
        if (!qsh) {  // set_history(None): forget the moments
            h->have_start = h->given = false;
            return;
        }
        h->start = moments_from(h->mol, qsh, dpat, qpat);
        h->have_start = true;
        h->given = given != 0;
    });
}

int axtb_gpu_batch_create(const AxtbMol* mols, int32_t nmol, const AxtbOptions* opts, AxtbBatch** out) {
    if (!out || !mols || nmol <= 0) return AXTB_ERR_INPUT;
    *out = nullptr;
    AxtbBatch* b = new AxtbBatch();
    int rc = guarded(nullptr, [&] {
        Opt o = to_opt(opts);
        check_options(o);
        vector<HostMol> v;
        v.reserve(nmol);
        for (int i = 0; i < nmol; i++) {
            try {
                v.push_back(to_mol(mols[i]));
            } catch (const Fail& f) {
                throw Fail(f.code, "molecule " + std::to_string(i) + ": " + f.what());
            }
        }
        b->build(v, o);
    });
    if (rc != AXTB_OK) {
        delete b;
        return rc;
    }
    *out = b;
    return AXTB_OK;
}

int axtb_gpu_batch_run(AxtbBatch* b, const double* positions, int32_t want_gradient, AxtbResult* outs, int32_t* status) {
    if (!b || !outs) return AXTB_ERR_INPUT;
    return guarded(&b->err, [&] {
        if (positions) {
            size_t off = 0;
            for (auto& m : b->mols) {
                m.xyz.assign(positions + off, positions + off + 3 * (size_t)m.nat);
                off += 3 * (size_t)m.nat;
            }
            b->upload_positions(positions, false);
        } else {
            vector<double> all;
            for (auto& m : b->mols) all.insert(all.end(), m.xyz.begin(), m.xyz.end());
            b->upload_positions(all.data(), false);
        }
        bool lv = std::any_of(outs, outs + b->nmol, [](const AxtbResult& r) { return r.emo || r.focc || r.focc_alpha; });
        b->run(want_gradient != 0, false, lv);
        b->extract(outs, status, want_gradient != 0);
    });
}

int axtb_gpu_batch_run_device(AxtbBatch* b, const double* d_positions, int32_t want_gradient, double* d_energy,
                              double* d_gradient, int32_t* status) {
    if (!b || !d_positions) return AXTB_ERR_INPUT;
    return guarded(&b->err, [&] {
        b->upload_positions(d_positions, true);
        b->run(want_gradient != 0);
        if (d_energy) {
            axg::k_total_energy<<<(b->nmol + 255) / 256, 256, 0, b->st>>>(b->nmol, b->S.e_fixed, b->d_eatm, b->S.energy,
                                                                           d_energy);
            b->launches++;
        }
        if (want_gradient && d_gradient)
            CK(cudaMemcpyAsync(d_gradient, b->S.grad, sizeof(double) * 3 * b->natT, cudaMemcpyDeviceToDevice, b->st));
        if (status) {
            vector<int> st_(b->nmol), conv(b->nmol);
            CK(cudaMemcpyAsync(st_.data(), b->S.status, sizeof(int) * b->nmol, cudaMemcpyDeviceToHost, b->st));
            CK(cudaMemcpyAsync(conv.data(), b->S.conv, sizeof(int) * b->nmol, cudaMemcpyDeviceToHost, b->st));
            CK(cudaStreamSynchronize(b->st));
            for (int m = 0; m < b->nmol; m++) status[m] = status_code(st_[m], conv[m]);
        }
    });
}

void* axtb_gpu_batch_stream(AxtbBatch* b) { return b ? (void*)b->st : nullptr; }

int64_t axtb_gpu_batch_launches(const AxtbBatch* b) { return b ? b->launches : 0; }

void axtb_gpu_batch_destroy(AxtbBatch* b) { delete b; }

int axtb_gpu_batch(const AxtbMol* mols, int32_t nmol, const AxtbOptions* opts, int32_t want_gradient, AxtbResult* outs,
                   int32_t* status) {
    AxtbBatch* b = nullptr;
    int rc = axtb_gpu_batch_create(mols, nmol, opts, &b);
    if (rc != AXTB_OK) return rc;
    rc = axtb_gpu_batch_run(b, nullptr, want_gradient, outs, status);
    axtb_gpu_batch_destroy(b);
    return rc;
}

// ---- introspection (include/axtb_gpu_debug.h)
int axtb_gpu_batch_set_restart(AxtbBatch* b, int32_t enable) {
    if (!b || enable < 0 || enable > 2) return AXTB_ERR_INPUT;
    return guarded(&b->err, [&] {
        b->restart = enable != 0;
        b->retry_fresh = enable != 2;
        CK(cudaMemsetAsync(b->S.have_guess, 0, sizeof(int) * b->nmol, b->st));
        CK(cudaStreamSynchronize(b->st));
    });
}

int axtb_gpu_batch_get_moments(AxtbBatch* b, int32_t mol, double* qsh, double* dpat, double* qpat) {
    if (!b || mol < 0 || mol >= b->nmol) return AXTB_ERR_INPUT;
    return guarded(&b->err, [&] {
        int conv = 0;
        CK(cudaMemcpyAsync(&conv, b->S.conv + mol, sizeof(int), cudaMemcpyDeviceToHost, b->st));
        CK(cudaStreamSynchronize(b->st));
        if (!conv) throw Fail(AXTB_ERR_INPUT, "molecule " + std::to_string(mol) + " has no converged moments");
        moments_to(b->get_moments(mol), qsh, dpat, qpat);
    });
}

int axtb_gpu_batch_set_moments(AxtbBatch* b, int32_t mol, const double* qsh, const double* dpat, const double* qpat) {
    if (!b || mol < 0 || mol >= b->nmol) return AXTB_ERR_INPUT;
    return guarded(&b->err, [&] {
        b->put_moments(mol, moments_from(b->mols[mol], qsh, dpat, qpat));
        int one = 1;
        CK(cudaMemcpyAsync(b->S.have_guess + mol, &one, sizeof(int), cudaMemcpyHostToDevice, b->st));
        CK(cudaStreamSynchronize(b->st));
        b->restart = true;
    });
}

int axtb_gpu_batch_set_profiling(AxtbBatch* b, int32_t enable) {
    if (!b) return AXTB_ERR_INPUT;
    b->profiling = enable != 0;
    b->prof.clear();
    for (double& c : b->team_cycles) c = 0.0;
    b->h2d_bytes = b->d2h_bytes = 0;
    return AXTB_OK;
}

int axtb_gpu_batch_profile(const AxtbBatch* b, char* buf, size_t len) {
    if (!b) return AXTB_ERR_INPUT;
    std::string s = "{\"kernels\": {";
    bool first = true;
    for (auto& kv : b->prof) {
        char tmp[256];
        std::snprintf(tmp, sizeof tmp, "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f, \"flops\": %.6e, \"bytes\": %.6e}",
                      first ? "" : ", ", kv.first.c_str(), kv.second.launches, kv.second.ms, kv.second.flops,
                      kv.second.bytes);
        s += tmp;
        first = false;
    }
    // SM-cycle shares of the eigen phase's parts (one-CTA teams)
    static const char* PH[8] = {"transform", "tridiagonal", "bisection", "fermi", "inverse_iteration",
                                "back_transform", "c_matrix", "density"};
    // slots 8..13: parts of the tridiagonal reduction (counted instead of slot 1)
    static const char* TP[6] = {"column_update", "householder", "symv", "panel_dots", "combine", "trailing_gemm"};
    // slots 16..19: the two-stage path's band reduction and bulge chasing (counted instead of
    // slot 1) and its Q2 and Q1 back-transformations (instead of slot 5)
    static const char* BP[4] = {"band_reduction", "bulge_chasing", "apply_q2", "apply_q1"};
    double ph[8], tc = 0.0, tt = 0.0;
    for (int k = 0; k < 8; k++) ph[k] = b->team_cycles[k];
    for (int k = 8; k < 14; k++) tt += b->team_cycles[k];
    ph[1] += tt + b->team_cycles[16] + b->team_cycles[17];
    ph[5] += b->team_cycles[18] + b->team_cycles[19];
    for (int k = 0; k < 8; k++) tc += ph[k];
    s += "}, \"team_eigen_phases\": {";
    for (int k = 0; k < 8; k++) {
        char tmp[96];
        std::snprintf(tmp, sizeof tmp, "%s\"%s\": %.4f", k ? ", " : "", PH[k], tc > 0 ? ph[k] / tc : 0.0);
        s += tmp;
    }
    s += "}, \"tridiagonal_parts\": {";
    for (int k = 0; k < 6; k++) {
        char tmp[96];
        std::snprintf(tmp, sizeof tmp, "%s\"%s\": %.4f", k ? ", " : "", TP[k],
                      tt > 0 ? b->team_cycles[8 + k] / tt : 0.0);
        s += tmp;
    }
    s += "}, \"two_stage_parts\": {";
    for (int k = 0; k < 4; k++) {
        char tmp[96];
        std::snprintf(tmp, sizeof tmp, "%s\"%s\": %.4f", k ? ", " : "", BP[k], tc > 0 ? b->team_cycles[16 + k] / tc : 0.0);
        s += tmp;
    }
    s += "}, \"eigen_launch_ms\": [";
    for (size_t k = 0; k < b->eigen_ms.size(); k++) {
        char tmp[32];
        std::snprintf(tmp, sizeof tmp, "%s%.3f", k ? ", " : "", b->eigen_ms[k]);
        s += tmp;
    }
    char tail[160];
    std::snprintf(tail, sizeof tail, "], \"h2d_bytes\": %lld, \"d2h_bytes\": %lld, \"grid\": %d}", b->h2d_bytes,
                  b->d2h_bytes, b->grid);
    s += tail;
    if (buf && len > 0) {
        size_t n = std::min(len - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return (int)s.size();
}

int axtb_gpu_batch_debug(AxtbBatch* b, int32_t mol, int32_t what, double* out) {
    if (!b || !out || mol < 0 || mol >= b->nmol) return AXTB_ERR_INPUT;
    return guarded(&b->err, [&] {
        int nat = b->mols[mol].nat, n = b->mols[mol].nao;
        long long a0 = b->m_at0[mol], o0 = b->m_ao0[mol], mat = b->m_mat0[mol], nn = b->nnT;
        auto cp = [&](const double* src, size_t cnt) {
            CK(cudaMemcpyAsync(out, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost, b->st));
        };
        size_t n2 = (size_t)n * n;
        switch (what) {
            case AXTB_DBG_CN: cp(b->S.cn + a0, nat); break;
            case AXTB_DBG_OVERLAP: cp(b->S.S + mat, n2); break;
            case AXTB_DBG_H0: cp(b->S.H0 + mat, n2); break;
            case AXTB_DBG_DIPOLE:
                for (int k = 0; k < 3; k++)
                    CK(cudaMemcpyAsync(out + k * n2, b->S.D + k * nn + mat, sizeof(double) * n2, cudaMemcpyDeviceToHost, b->st));
                break;
            case AXTB_DBG_QUADRUPOLE:
                for (int k = 0; k < 6; k++)
                    CK(cudaMemcpyAsync(out + k * n2, b->S.Q + k * nn + mat, sizeof(double) * n2, cudaMemcpyDeviceToHost, b->st));
                break;
            case AXTB_DBG_DENSITY: cp(b->S.P + mat, n2); break;
            case AXTB_DBG_FOCK: cp(b->S.F + mat, n2); break;
            case AXTB_DBG_EMO: cp(b->S.emo + o0, n); break;
            case AXTB_DBG_FOCC: cp(b->S.focc + o0, n); break;
            case AXTB_DBG_WDENSITY: cp(b->S.W + mat, n2); break;
            case AXTB_DBG_EEQ: cp(b->P.eeq_q + a0, nat); break;
            case AXTB_DBG_LINV: cp(b->S.Linv + mat, n2); break;
            case AXTB_DBG_EIGEN_CYCLES: cp(b->S.mol_cyc + mol, 1); break;
            case AXTB_DBG_STATUS_BITS: {
                int bits = 0;
                CK(cudaMemcpyAsync(&bits, b->S.status + mol, sizeof(int), cudaMemcpyDeviceToHost, b->st));
                CK(cudaStreamSynchronize(b->st));
                *out = (double)bits;
                break;
            }
            default: throw Fail(AXTB_ERR_INPUT, "unknown debug quantity");
        }
        CK(cudaStreamSynchronize(b->st));
    });
}

}  // extern "C"
