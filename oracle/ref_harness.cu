// ref_harness.cu -- TEST INFRASTRUCTURE ONLY. A C-callable harness around the reference's own,
// unmodified dom::DOM (K3DOM, or DS-PHD/MIB with -DREF_DS), compiled from its sources together
// with this file by oracle/build_ref.sh into oracle/_ref/. The tests use it to run the
// reference's public stage methods (include/common/dom.h:89-94, include/k3dom/dom.h:23-29,
// include/dsphdmib/dom.h:23-32) on states and draws identical to those fed to the library.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <thrust/binary_search.h>
#include <thrust/device_vector.h>
#include <thrust/scan.h>

#include <vector>

#include "common/dom_types.h"
#include "common/kernel/init.h"
#ifdef REF_DS
#include "dsphdmib/dom.h"
#else
#include "k3dom/dom.h"
#endif

namespace {

struct RefDOM : public dom::DOM {
    explicit RefDOM(const Params& p) : dom::DOM(p) {}
    void set_time(float t) { updated_time = t; }
    float get_time() const { return updated_time; }
    void bump_iteration() { iteration++; }
    void sensor_rel(float* s) const {
        s[0] = sensor_pos_x - center_pos_x;
        s[1] = sensor_pos_y - center_pos_y;
        s[2] = sensor_pos_z - center_pos_z;
    }
    int states() const { return (int)(particles_grid.x * block_dim.x); }
};

__global__ void set_states(curandState* s, int n, unsigned long long seed, unsigned frame, unsigned stage,
                           unsigned dpi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    s[i].seed = seed;
    s[i].tid = (unsigned)i;
    s[i].calls = 0;
    s[i].stage = stage;
    s[i].frame = frame;
    s[i].dpi = dpi;
}

void zero_soa(dom::ParticlesSoA& a) {
    cudaMemset(a.state_pos, 0, a.size * sizeof(glm::vec3));
    cudaMemset(a.state_vel, 0, a.size * sizeof(glm::vec3));
    cudaMemset(a.grid_cell_idx, 0, a.size * sizeof(int));
    cudaMemset(a.weight, 0, a.size * sizeof(float));
    cudaMemset(a.post_weight, 0, a.size * sizeof(float));
    cudaMemset(a.associated, 0, a.size * sizeof(bool));
}

dom::ParticlesSoA* pick(RefDOM* d, int which) {
    return which == 0 ? &d->particle_array : (which == 1 ? &d->particle_array_next : &d->birth_particle_array);
}

struct Draws {
    unsigned long long seed;
    unsigned frame;
};

}  // namespace

extern "C" {

// params: a dom::DOM_c::Params laid out as k3dom_params' leading fields.
void* ref_create(const void* params, unsigned long long seed) {
    dom::DOM_c::Params p;
    memcpy(&p, params, sizeof(p));
    RefDOM* d = new RefDOM(p);
    cudaDeviceSynchronize();
    // deterministic start: the reference leaves particle memory uninitialised
    zero_soa(d->particle_array);
    zero_soa(d->particle_array_next);
    zero_soa(d->birth_particle_array);
    cudaMemset(d->grid_cell_array, 0, sizeof(dom::GridCell) * d->grid_cell_count);
    cudaMemset(d->born_masses_array, 0, sizeof(float) * d->grid_cell_count);
    dom::initGridCellsKernel<<<d->grid_map_grid, d->block_dim>>>(d->grid_cell_array, d->grid_size, d->grid_cell_count,
                                                                 p.prior_free, p.prior_static, p.prior_dynamic,
                                                                 p.prior_occ);
    cudaDeviceSynchronize();
    (void)seed;
    return d;
}

void ref_destroy(void* h) {
    delete static_cast<RefDOM*>(h);
    cudaDeviceSynchronize();
}

int ref_last_error(void) { return (int)cudaGetLastError(); }

void ref_sizes(void* h, int* out) {
    RefDOM* d = static_cast<RefDOM*>(h);
    out[0] = d->grid_size;
    out[1] = d->grid_size_z;
    out[2] = d->grid_cell_count;
    out[3] = d->particle_count;
    out[4] = d->new_born_particle_count;
    out[5] = d->states();
}

void ref_update_pose(void* h, float x, float y, float z) { static_cast<RefDOM*>(h)->updatePose(x, y, z); }

void ref_sensor_rel(void* h, float* s) { static_cast<RefDOM*>(h)->sensor_rel(s); }

// DOM_c::getCenterPosition{X,Y,Z} (include/common/dom.h:62-64): the map centre that updatePose's
// shift rule moves (src/common/dom.cu:125-154).
void ref_center(void* h, float* c) {
    RefDOM* d = static_cast<RefDOM*>(h);
    c[0] = d->getCenterPositionX();
    c[1] = d->getCenterPositionY();
    c[2] = d->getCenterPositionZ();
}

// DOM_c::indexToCoord{X,Y,Z} (include/common/dom.h:70-81) for n cell indices, host side, as the
// node's publish_mapdata calls them (src/k3dom/k3dom_node.cpp:166-168).
void ref_index_to_coord(void* h, const int* idx, long long n, float* xyz) {
    RefDOM* d = static_cast<RefDOM*>(h);
    for (long long k = 0; k < n; ++k) {
        xyz[3 * k + 0] = d->indexToCoordX(idx[k]);
        xyz[3 * k + 1] = d->indexToCoordY(idx[k]);
        xyz[3 * k + 2] = d->indexToCoordZ(idx[k]);
    }
}

void ref_set_draws(void* h, unsigned long long seed, unsigned frame, unsigned stage, unsigned dpi) {
    RefDOM* d = static_cast<RefDOM*>(h);
    const int n = d->states();
    set_states<<<(n + 255) / 256, 256>>>(d->rng_states, n, seed, frame, stage, dpi);
    cudaDeviceSynchronize();
}

void ref_particle_prediction(void* h, float dt) {
    static_cast<RefDOM*>(h)->particlePrediction(dt);
    cudaDeviceSynchronize();
}

void ref_particle_assignment(void* h) {
    static_cast<RefDOM*>(h)->particleAssignment();
    cudaDeviceSynchronize();
}

void ref_occupancy(void* h, float dt, const float* xs, const float* ys, const float* zs, int n) {
    std::vector<float> x(xs, xs + n), y(ys, ys + n), z(zs, zs + n);
#ifdef REF_DS
    (void)dt;
    static_cast<RefDOM*>(h)->gridCellOccupancyUpdate(x, y, z);
#else
    static_cast<RefDOM*>(h)->gridCellOccupancyUpdate(dt, x, y, z);
#endif
    cudaDeviceSynchronize();
}

void ref_update_persistent(void* h) {
    static_cast<RefDOM*>(h)->updatePersistentParticles();
    cudaDeviceSynchronize();
}

void ref_initialize_new_particles(void* h) {
    static_cast<RefDOM*>(h)->initializeNewParticles();
    cudaDeviceSynchronize();
}

void ref_statistical_moments(void* h) {
    static_cast<RefDOM*>(h)->statisticalMoments();
    cudaDeviceSynchronize();
}

void ref_resampling(void* h) {
    static_cast<RefDOM*>(h)->resampling();
    cudaDeviceSynchronize();
}

void ref_initialize_particles(void* h, const float* xs, const float* ys, const float* zs, int n) {
    std::vector<float> x(xs, xs + n), y(ys, ys + n), z(zs, zs + n);
    static_cast<RefDOM*>(h)->initializeParticles(x, y, z);
    cudaDeviceSynchronize();
}

// The tail of updateGrid (src/k3dom/dom.cu:43-49): particle_array = particle_array_next.
void ref_finish(void* h, float t, int was_steady) {
    RefDOM* d = static_cast<RefDOM*>(h);
    if (was_steady) d->particle_array = d->particle_array_next;
    cudaDeviceSynchronize();
    d->set_time(t);
#ifdef REF_DS
    d->bump_iteration();
#endif
}

// The reference's own updateGrid, used for timing (draws from whatever stage the states hold).
void ref_update_grid(void* h, float t, const float* xs, const float* ys, const float* zs, int n) {
    std::vector<float> x(xs, xs + n), y(ys, ys + n), z(zs, zs + n);
    static_cast<RefDOM*>(h)->updateGrid(t, x, y, z);
}

float ref_updated_time(void* h) { return static_cast<RefDOM*>(h)->get_time(); }

// which: 0 = particle_array, 1 = particle_array_next, 2 = birth_particle_array.
void ref_get_particles(void* h, int which, float* pos, float* vel, float* w, int* cell, unsigned char* assoc) {
    dom::ParticlesSoA* a = pick(static_cast<RefDOM*>(h), which);
    const size_t n = a->size;
    if (pos) cudaMemcpy(pos, a->state_pos, n * sizeof(glm::vec3), cudaMemcpyDeviceToHost);
    if (vel) cudaMemcpy(vel, a->state_vel, n * sizeof(glm::vec3), cudaMemcpyDeviceToHost);
    if (w) cudaMemcpy(w, a->weight, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (cell) cudaMemcpy(cell, a->grid_cell_idx, n * sizeof(int), cudaMemcpyDeviceToHost);
    if (assoc) cudaMemcpy(assoc, a->associated, n * sizeof(bool), cudaMemcpyDeviceToHost);
}

void ref_set_particles(void* h, int which, const float* pos, const float* vel, const float* w, const int* cell,
                       const unsigned char* assoc) {
    dom::ParticlesSoA* a = pick(static_cast<RefDOM*>(h), which);
    const size_t n = a->size;
    if (pos) cudaMemcpy(a->state_pos, pos, n * sizeof(glm::vec3), cudaMemcpyHostToDevice);
    if (vel) cudaMemcpy(a->state_vel, vel, n * sizeof(glm::vec3), cudaMemcpyHostToDevice);
    if (w) cudaMemcpy(a->weight, w, n * sizeof(float), cudaMemcpyHostToDevice);
    if (cell) cudaMemcpy(a->grid_cell_idx, cell, n * sizeof(int), cudaMemcpyHostToDevice);
    if (assoc) cudaMemcpy(a->associated, assoc, n * sizeof(bool), cudaMemcpyHostToDevice);
}

// 68-byte dom::GridCell records.
void ref_get_cells(void* h, void* out) {
    RefDOM* d = static_cast<RefDOM*>(h);
    cudaMemcpy(out, d->grid_cell_array, sizeof(dom::GridCell) * d->grid_cell_count, cudaMemcpyDeviceToHost);
}

void ref_set_cells(void* h, const void* in) {
    RefDOM* d = static_cast<RefDOM*>(h);
    cudaMemcpy(d->grid_cell_array, in, sizeof(dom::GridCell) * d->grid_cell_count, cudaMemcpyHostToDevice);
}

void ref_get_born(void* h, float* out) {
    RefDOM* d = static_cast<RefDOM*>(h);
    cudaMemcpy(out, d->born_masses_array, sizeof(float) * d->grid_cell_count, cudaMemcpyDeviceToHost);
}

void ref_set_born(void* h, const float* in) {
    RefDOM* d = static_cast<RefDOM*>(h);
    cudaMemcpy(d->born_masses_array, in, sizeof(float) * d->grid_cell_count, cudaMemcpyHostToDevice);
}

#ifdef REF_DS
void ref_get_meas(void* h, float* occ, float* fr) {
    RefDOM* d = static_cast<RefDOM*>(h);
    std::vector<dom::MeasurementCell> m(d->grid_cell_count);
    cudaMemcpy(m.data(), d->meas_cell_array, sizeof(dom::MeasurementCell) * d->grid_cell_count,
               cudaMemcpyDeviceToHost);
    for (int i = 0; i < d->grid_cell_count; ++i) {
        occ[i] = m[i].occ_mass;
        fr[i] = m[i].free_mass;
    }
}
#endif

// The library calls the reference makes, run on given arrays: thrust::inclusive_scan
// (include/common/common.h:7-18) and thrust::lower_bound (resampling.cu:66-67).
void ref_thrust_scan(const float* in, long long n, float* out) {
    thrust::device_vector<float> a(in, in + n), r(n);
    thrust::inclusive_scan(a.begin(), a.end(), r.begin());
    cudaMemcpy(out, thrust::raw_pointer_cast(r.data()), sizeof(float) * n, cudaMemcpyDeviceToHost);
}

void ref_thrust_lower_bound(const float* cum, long long n, const float* u, long long m, int* out) {
    thrust::device_vector<float> a(cum, cum + n), b(u, u + m);
    thrust::device_vector<int> r(m);
    thrust::lower_bound(a.begin(), a.end(), b.begin(), b.end(), r.begin());
    cudaMemcpy(out, thrust::raw_pointer_cast(r.data()), sizeof(int) * m, cudaMemcpyDeviceToHost);
}

}  // extern "C"
