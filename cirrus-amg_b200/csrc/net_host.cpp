// Host side of the learned finest-level smoother's network: parameters, Adam state,
// training samples and the training loop, all on the device (kernels in learned.cu).
#include <cmath>
#include <cstring>
#include <vector>

#include "cmg_impl.hpp"

namespace cmg {

namespace {

#define NCK(call)                                     \
    do {                                              \
        int _rc = check_cuda((call), #call);          \
        if (_rc) return _rc;                          \
    } while (0)

template <class T>
void nfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number generators", 2014)
struct SplitMix {
    unsigned long long s;
    unsigned long long next() {
        unsigned long long z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }  // (0, 1)
    double normal() {  // Box-Muller
        const double u = uniform(), v = uniform();
        return std::sqrt(-2.0 * std::log(u)) * std::cos(6.283185307179586 * v);
    }
};

}  // namespace

Net::~Net() {
    nfree(p);
    nfree(m);
    nfree(v);
    nfree(pack);
    nfree(bias);
    nfree(rho);
    nfree(diag);
    nfree(types);
    nfree(target);
    nfree(faces);
    nfree(halo);
    nfree(grad);
    nfree(loss);
    nfree(gsum);
    nfree(idx);
    if (scratch) cudaFree(scratch);
    if (st) cudaStreamDestroy(st);
}

// He-normal weights (fan-in 27 x used input channels), zero biases, a small last layer so
// that the untrained smoother starts close to the plain cycle
int Net::init(int hidden, unsigned long long seed) {
    static const bool ok = net_init();
    if (!ok) {
        set_error("learned: the network kernels cannot be configured on this device");
        return 2;
    }
    if (hidden == 32) {
        static const bool deep_ok = deep_init();
        if (!deep_ok) {
            set_error("learned: the residual network's kernels cannot be configured on this device");
            return 2;
        }
    }
    H = hidden;
    np = net_params(H);
    NCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    NCK(cudaMalloc(&p, sizeof(float) * np));
    NCK(cudaMalloc(&m, sizeof(float) * np));
    NCK(cudaMalloc(&v, sizeof(float) * np));
    NCK(cudaMalloc(&gsum, sizeof(float) * np));
    NCK(cudaMalloc(&pack, sizeof(uint16_t) * (size_t)net_pack_elems(H)));
    NCK(cudaMalloc(&bias, sizeof(float) * net_bias_elems(H)));
    std::vector<float> h(np, 0.0f);
    SplitMix rng{seed};
    if (H == 32) {
        // residual net: He-normal W0 (7 feature channels in use) and Wa; Wb at a tenth of He so
        // that each block starts close to the identity; zero biases; a small output layer
        const int C = 32, blk = 2 * C * 27 * C + 2 * C, wo = C * 216 + C + 4 * blk;
        const double s0 = std::sqrt(2.0 / (27.0 * 7.0)), sh = std::sqrt(2.0 / (27.0 * C)), so = 0.1 * std::sqrt(1.0 / (27.0 * C));
        for (int n = 0; n < C; ++n)
            for (int t = 0; t < 27; ++t)
                for (int c = 0; c < 8; ++c) h[(n * 27 + t) * 8 + c] = c < 7 ? (float)(s0 * rng.normal()) : 0.0f;
        for (int k = 0; k < 4; ++k) {
            const int wa = C * 216 + C + k * blk, wb = wa + C * 27 * C + C;
            for (int e = 0; e < C * 27 * C; ++e) h[wa + e] = (float)(sh * rng.normal());
            for (int e = 0; e < C * 27 * C; ++e) h[wb + e] = (float)(0.1 * sh * rng.normal());
        }
        for (int e = wo; e < np; ++e) h[e] = (float)(so * rng.normal());
        return set_params(h.data());
    }
    const int w1 = 0, b1 = w1 + H * 216, w2 = b1 + H, b2 = w2 + H * 27 * H, w3 = b2 + H;
    const double s1 = std::sqrt(2.0 / (27.0 * 4.0)), s2 = std::sqrt(2.0 / (27.0 * H)), s3 = 0.1 * std::sqrt(1.0 / (27.0 * H));
    for (int n = 0; n < H; ++n)
        for (int t = 0; t < 27; ++t)
            for (int c = 0; c < 8; ++c) h[w1 + (n * 27 + t) * 8 + c] = c < 4 ? (float)(s1 * rng.normal()) : 0.0f;
    for (int e = w2; e < b2; ++e) h[e] = (float)(s2 * rng.normal());
    for (int e = w3; e < np; ++e) h[e] = (float)(s3 * rng.normal());
    (void)b1;
    return set_params(h.data());
}

int Net::set_params(const float* host) {
    NCK(cudaMemcpyAsync(p, host, sizeof(float) * np, cudaMemcpyHostToDevice, st));
    NCK(cudaMemsetAsync(m, 0, sizeof(float) * np, st));
    NCK(cudaMemsetAsync(v, 0, sizeof(float) * np, st));
    adam_step = 0;
    launch_net_pack(H, p, pack, bias, st);
    NCK(cudaStreamSynchronize(st));
    return 0;
}

int Net::get_params(float* host) {
    NCK(cudaMemcpyAsync(host, p, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
    return 0;
}

int Net::set_samples(int n, const float* hr, const float* hd, const uint8_t* ht, const float* htg, const float* hfaces, const float* hhalo) {
    nfree(rho);
    nfree(diag);
    nfree(types);
    nfree(target);
    nfree(loss);
    nfree(idx);
    nfree(faces);
    nfree(halo);
    ns = 0;
    if (n <= 0) return 0;
    const size_t c = (size_t)n * kCells;
    if (hfaces) {
        NCK(cudaMalloc(&faces, sizeof(float) * 3 * c));
        NCK(cudaMemcpyAsync(faces, hfaces, sizeof(float) * 3 * c, cudaMemcpyHostToDevice, st));
    }
    if (hhalo) {
        NCK(cudaMalloc(&halo, sizeof(float) * 768 * (size_t)n));
        NCK(cudaMemcpyAsync(halo, hhalo, sizeof(float) * 768 * (size_t)n, cudaMemcpyHostToDevice, st));
    }
    NCK(cudaMalloc(&rho, sizeof(float) * c));
    NCK(cudaMalloc(&diag, sizeof(float) * c));
    NCK(cudaMalloc(&types, c));
    NCK(cudaMalloc(&target, sizeof(float) * c));
    NCK(cudaMalloc(&loss, sizeof(float) * n));
    NCK(cudaMalloc(&idx, sizeof(int) * n));
    NCK(cudaMemcpyAsync(rho, hr, sizeof(float) * c, cudaMemcpyHostToDevice, st));
    NCK(cudaMemcpyAsync(diag, hd, sizeof(float) * c, cudaMemcpyHostToDevice, st));
    NCK(cudaMemcpyAsync(types, ht, c, cudaMemcpyHostToDevice, st));
    if (htg) NCK(cudaMemcpyAsync(target, htg, sizeof(float) * c, cudaMemcpyHostToDevice, st));
    else NCK(cudaMemsetAsync(target, 0, sizeof(float) * c, st));
    NCK(cudaStreamSynchronize(st));
    ns = n;
    return 0;
}

int Net::ensure_batch(int nb) {
    if (nb <= batch_cap) return 0;
    nfree(grad);
    if (scratch) cudaFree(scratch);
    scratch = nullptr;
    batch_cap = 0;
    NCK(cudaMalloc(&grad, sizeof(float) * (size_t)net_train_rows(H, nb) * np));
    if (const size_t sb = net_train_scratch_bytes(H, nb)) {
        // the activation planes' borders are never written: they stay zero
        NCK(cudaMalloc(&scratch, sb));
        NCK(cudaMemsetAsync(scratch, 0, sb, st));
    }
    batch_cap = nb;
    return 0;
}

// the samples' optional inputs from sample `first` on: faces [sample][3][512], halo [sample][768]
NetExtra Net::extra(int first) const {
    NetExtra ex;
    if (faces) {
        ex.faces = faces + (size_t)first * 3 * kCells;
        ex.fstride = kCells;
        ex.ftile = 3 * kCells;
    }
    if (halo) ex.halo = halo + (size_t)first * 768;
    return ex;
}

int Net::forward(int first, int n, float* out_host) {
    const size_t o = (size_t)first * kCells, c = (size_t)n * kCells;
    float* out = nullptr;
    NCK(cudaMalloc(&out, sizeof(float) * c));
    launch_net_forward(H, rho + o, nullptr, diag + o, types + o, nullptr, 0, n, pack, bias, out, true, st, extra(first));
    int rc = check_cuda(cudaMemcpyAsync(out_host, out, sizeof(float) * c, cudaMemcpyDeviceToHost, st), "forward: read-back");
    if (!rc) rc = check_cuda(cudaStreamSynchronize(st), "forward");
    cudaFree(out);
    if (!rc && net_take_tc_error() == 1) {
        set_error("learned forward: a tensor-core MMA did not complete in time");
        rc = 2;
    }
    return rc;
}

// loss = sum over samples of the tile loss (loss_kind) / (n * 512) and its gradient
int Net::gradient(int first, int n, double* loss_out, float* grad_host) {
    if (int rc = ensure_batch(n)) return rc;
    const size_t o = (size_t)first * kCells;
    launch_net_train(H, rho + o, diag + o, types + o, target + o, nullptr, n, pack, bias, grad, loss, loss_kind, st, extra(first), scratch);
    const float scale = 1.0f / ((float)n * kCells);
    launch_net_reduce_adam(grad, net_train_rows(H, n), np, scale, gsum, p, m, v, 0.0f, 0, false, st);
    if (net_take_tc_error() == 1) {
        set_error("learned gradient: a tensor-core MMA or bulk copy did not complete in time");
        return 2;
    }
    std::vector<float> l(n);
    NCK(cudaMemcpyAsync(l.data(), loss, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    if (grad_host) NCK(cudaMemcpyAsync(grad_host, gsum, sizeof(float) * np, cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
    double s = 0.0;
    for (float x : l) s += x;
    if (loss_out) *loss_out = s * scale;
    return 0;
}

// Adam over shuffled mini-batches; epoch_loss[e] = mean loss of epoch e's batches
int Net::train(int epochs, int batch, float lr, unsigned long long seed, float* epoch_loss) {
    if (ns <= 0) {
        set_error("learned train: no samples");
        return 3;
    }
    if (batch > ns) batch = ns;
    if (int rc = ensure_batch(batch)) return rc;
    SplitMix rng{seed};
    std::vector<int> perm(ns);
    std::vector<float> l(ns);
    for (int e = 0; e < epochs; ++e) {
        for (int i = 0; i < ns; ++i) perm[i] = i;
        for (int i = ns - 1; i > 0; --i) {  // Fisher-Yates
            const int j = (int)(rng.next() % (unsigned long long)(i + 1));
            std::swap(perm[i], perm[j]);
        }
        NCK(cudaMemcpyAsync(idx, perm.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
        for (int b0 = 0; b0 < ns; b0 += batch) {
            const int nb = ns - b0 < batch ? ns - b0 : batch;
            launch_net_train(H, rho, diag, types, target, idx + b0, nb, pack, bias, grad, loss + b0, loss_kind, st, extra(0), scratch);
            launch_net_reduce_adam(grad, net_train_rows(H, nb), np, 1.0f / ((float)nb * kCells), nullptr, p, m, v, lr, ++adam_step, true,
                                   st);
            launch_net_pack(H, p, pack, bias, st);
        }
        NCK(cudaMemcpyAsync(l.data(), loss, sizeof(float) * ns, cudaMemcpyDeviceToHost, st));
        NCK(cudaStreamSynchronize(st));
        if (net_take_tc_error() == 1) {
            set_error("learned train: a tensor-core MMA or bulk copy did not complete in time");
            return 2;
        }
        double s = 0.0;
        for (int i = 0; i < ns; ++i) s += l[i];
        if (epoch_loss) epoch_loss[e] = (float)(s / ((double)ns * kCells));
    }
    NCK(cudaGetLastError());
    return 0;
}

}  // namespace cmg
