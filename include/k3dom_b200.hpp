/*
 * k3dom_b200.hpp -- the reference's C++ interface, dom::DOM_c / dom::DOM
 * (include/common/dom.h:16-148, include/k3dom/dom.h:17-30, include/dsphdmib/dom.h:17-37), as a
 * header-only class over the C ABI of libk3dom_b200.so (k3dom_b200.h).
 *
 * Code written against the reference compiles against this header unchanged where it uses:
 *  - dom::DOM::Params (the same 26 fields; the library's additions seed and max_points are
 *    value-initialised to 0, i.e. seed 0 and the default point capacity);
 *  - DOM(const Params&), updatePose(x, y, z), updateGrid(t, xs, ys, zs), the public stage
 *    methods (particlePrediction, particleAssignment, gridCellOccupancyUpdate,
 *    updatePersistentParticles, initializeNewParticles, statisticalMoments, resampling,
 *    initializeParticles);
 *  - getGridSize, getResolution, getCenterPosition{X,Y,Z}, getSensorPosition{X,Y,Z},
 *    indexToCoord{X,Y,Z}, getIteration;
 *  - grid_cell_array (device, 68-byte dom::GridCell records), grid_cell_array_host (host, the
 *    caller's cudaMemcpy target, as in k3dom_node.cpp:131-132) and grid_cell_count, plus the
 *    GridCell helpers occ_mean, dyn_mean, total_mass, calcVar, occ_prob, mean_vel_sq
 *    (include/common/dom_types.h:47-64).
 *
 * Differences: failures throw dom::Error (the reference prints and continues); the variant is
 * chosen by defining K3DOM_B200_DSPHDMIB before including this header (the reference builds one
 * binary per variant because both classes are named dom::DOM), or per object through the
 * constructor's variant argument; grid_cell_array is refreshed from the library's cell state
 * after every call that changes it (the library keeps its cells as structure-of-arrays).
 */
#ifndef K3DOM_B200_HPP
#define K3DOM_B200_HPP

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "k3dom_b200.h"

namespace dom {

/* The reference's per-voxel record (include/common/dom_types.h:12-45): 68 bytes, same field
 * order, with its derived quantities (:47-64) evaluated in FP32 as written there. */
struct GridCell {
    int start_idx;
    int end_idx;
    float mu_A;
    float mu_UA;
    float w_A;
    float w_UA;
    float mean_x_vel;
    float mean_y_vel;
    float mean_z_vel;
    float likelihood;
    float p_A;
    float free_mass;
    float static_mass;
    float dynamic_mass;
    float occ_mass;
    float pers_mass;
    float pred_mass;

    float total_mass() const { return free_mass + static_mass + dynamic_mass; }
    float occ_mean() const { return (static_mass + dynamic_mass) / total_mass(); }
    float dyn_mean() const { return dynamic_mass / total_mass(); }
    float calcVar() const {
        const float sum = total_mass();
        if (sum == 0.0f) return 1e6f;
        float top = free_mass > static_mass ? free_mass : static_mass;
        top = top > dynamic_mass ? top : dynamic_mass;
        const float mean = top / sum;
        return mean * (1.0f - mean) / (sum + 1.0f);
    }
    float occ_prob() const { return occ_mass + (1.0f - occ_mass - free_mass) / 2.0f; }
    float mean_vel_sq() const {
        return mean_x_vel * mean_x_vel + mean_y_vel * mean_y_vel + mean_z_vel * mean_z_vel;
    }
};
static_assert(sizeof(GridCell) == K3DOM_GRIDCELL_BYTES, "dom::GridCell must keep the reference's 68-byte layout");

/* The /map_data point of k3dom_node.cpp:161-184 (include/common/mappoint.h:5-28) without PCL's
 * alignment padding: the layout k3dom_get_mappoints writes. */
struct MapPoint {
    float x, y, z, v_x, v_y, v_z, occ_val, dyn_val, eval_aug, dyn_aug;
};
static_assert(sizeof(MapPoint) == K3DOM_MAPPOINT_FLOATS * sizeof(float), "MapPoint layout");

class Error : public std::runtime_error {
public:
    Error(const std::string& what, k3dom_status s)
        : std::runtime_error(what + ": " + k3dom_status_string(s)), status(s) {}
    k3dom_status status;
};

inline void check(k3dom_status s, const char* what) {
    if (s != K3DOM_OK) throw Error(what, s);
}

#ifdef K3DOM_B200_DSPHDMIB
constexpr k3dom_variant kDefaultVariant = K3DOM_VARIANT_DSPHDMIB;
#else
constexpr k3dom_variant kDefaultVariant = K3DOM_VARIANT_K3DOM;
#endif

class DOM_c {
public:
    /* dom::DOM_c::Params (include/common/dom.h:19-52): the same fields, in the same order; the
     * library's trailing additions start at zero. */
    struct Params : k3dom_params {
        Params() : k3dom_params() {}
    };

    explicit DOM_c(const Params& params, k3dom_variant variant = kDefaultVariant, int device = 0)
        : params(params), variant_(variant) {
        check(k3dom_create(&params, variant, device, &h_), "k3dom_create");
        k3dom_info i{};
        check(k3dom_get_info(h_, &i), "k3dom_get_info");
        grid_size = i.grid_size;
        grid_size_z = i.grid_size_z;
        grid_cell_count = i.grid_cell_count;
        particle_count = i.particle_count;
        new_born_particle_count = i.new_born_particle_count;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        const size_t bytes = sizeof(GridCell) * (size_t)grid_cell_count;
        cudaError_t e = cudaMalloc(&grid_cell_array, bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&grid_cell_array_host, bytes);
        cudaSetDevice(prev);
        if (e != cudaSuccess) {
            release();
            throw Error("allocating grid_cell_array", K3DOM_ERR_OUT_OF_MEMORY);
        }
        refresh();
    }
    DOM_c(const DOM_c&) = delete;
    DOM_c& operator=(const DOM_c&) = delete;
    virtual ~DOM_c() { release(); }

    /* DOM_c::updatePose (src/common/dom.cu:111-158). */
    void updatePose(float new_x, float new_y, float new_z) {
        check(k3dom_update_pose(h_, new_x, new_y, new_z), "updatePose");
        refresh();
    }

    int getGridSize() const { return grid_size; }
    float getResolution() const { return params.resolution; }
    float getCenterPositionX() const { return info().center_x; }
    float getCenterPositionY() const { return info().center_y; }
    float getCenterPositionZ() const { return info().center_z; }
    float getSensorPositionX() const { return info().sensor_x; }
    float getSensorPositionY() const { return info().sensor_y; }
    float getSensorPositionZ() const { return info().sensor_z; }
    float indexToCoordX(int i) const { return coord(i, 0); }
    float indexToCoordY(int i) const { return coord(i, 1); }
    float indexToCoordZ(int i) const { return coord(i, 2); }
    int getIteration() const { return info().iteration; }

    /* Public stage methods (include/common/dom.h:89-94). */
    void particlePrediction(float dt) { stage(k3dom_particle_prediction(h_, dt), "particlePrediction"); }
    void particleAssignment() { stage(k3dom_particle_assignment(h_), "particleAssignment"); }
    void updatePersistentParticles() {
        stage(k3dom_update_persistent_particles(h_), "updatePersistentParticles");
    }
    void initializeNewParticles() { stage(k3dom_initialize_new_particles(h_), "initializeNewParticles"); }
    void statisticalMoments() { stage(k3dom_statistical_moments(h_), "statisticalMoments"); }
    void resampling() { stage(k3dom_resampling(h_), "resampling"); }

    /* The node's readback (k3dom_node.cpp:131-132) in one call: grid_cell_array_host <- cells. */
    void copyGridCellsToHost() {
        check(k3dom_get_gridcell_aos(h_, grid_cell_array_host, K3DOM_MEM_HOST), "k3dom_get_gridcell_aos");
    }
    /* The /map_data cloud (k3dom_node.cpp:161-184), grid_cell_count points. */
    std::vector<MapPoint> mapPoints() const {
        std::vector<MapPoint> out((size_t)grid_cell_count);
        check(k3dom_get_mappoints(h_, reinterpret_cast<float*>(out.data()), K3DOM_MEM_HOST), "k3dom_get_mappoints");
        return out;
    }

    k3dom_handle* handle() const { return h_; }
    k3dom_variant variant() const { return variant_; }

    Params params;
    GridCell* grid_cell_array = nullptr;       /* device: the cells after the last call */
    GridCell* grid_cell_array_host = nullptr;  /* host (pinned): the caller's readback target */
    int grid_size = 0;
    int grid_size_z = 0;
    int grid_cell_count = 0;
    int particle_count = 0;
    int new_born_particle_count = 0;

protected:
    k3dom_info info() const {
        k3dom_info i{};
        check(k3dom_get_info(h_, &i), "k3dom_get_info");
        return i;
    }
    float coord(int idx, int axis) const {
        float xyz[3];
        check(k3dom_index_to_coord(h_, idx, &xyz[0], &xyz[1], &xyz[2]), "k3dom_index_to_coord");
        return xyz[axis];
    }
    void refresh() {
        check(k3dom_get_gridcell_aos(h_, grid_cell_array, K3DOM_MEM_DEVICE), "k3dom_get_gridcell_aos");
    }
    void stage(k3dom_status s, const char* what) {
        check(s, what);
        refresh();
    }
    static void points(const std::vector<float>& xs, const std::vector<float>& ys, const std::vector<float>& zs) {
        if (xs.size() != ys.size() || xs.size() != zs.size())  // src/k3dom/dom.cu:83 asserts this
            throw Error("measurement vectors differ in length", K3DOM_ERR_INVALID_ARGUMENT);
    }
    void release() {
        if (grid_cell_array) cudaFree(grid_cell_array);
        if (grid_cell_array_host) cudaFreeHost(grid_cell_array_host);
        grid_cell_array = nullptr;
        grid_cell_array_host = nullptr;
        if (h_) k3dom_destroy(h_);
        h_ = nullptr;
    }

    k3dom_handle* h_ = nullptr;
    k3dom_variant variant_;
};

class DOM : public DOM_c {
public:
    explicit DOM(const Params& params, k3dom_variant variant = kDefaultVariant, int device = 0)
        : DOM_c(params, variant, device) {}

    /* DOM::updateGrid (src/k3dom/dom.cu:29-50, src/dsphdmib/dom.cu:32-53): points are metres,
     * sensor-centred and map-axis aligned; returns when the frame is complete. */
    void updateGrid(float t, const std::vector<float>& measurements_x, const std::vector<float>& measurements_y,
                    const std::vector<float>& measurements_z) {
        points(measurements_x, measurements_y, measurements_z);
        stage(k3dom_update_grid(h_, t, measurements_x.data(), measurements_y.data(), measurements_z.data(),
                                (int32_t)measurements_x.size(), K3DOM_MEM_HOST),
              "updateGrid");
    }
    /* DOM::initializeParticles (src/k3dom/dom.cu:52-77). */
    void initializeParticles(const std::vector<float>& measurements_x, const std::vector<float>& measurements_y,
                             const std::vector<float>& measurements_z) {
        points(measurements_x, measurements_y, measurements_z);
        stage(k3dom_initialize_particles(h_, measurements_x.data(), measurements_y.data(), measurements_z.data(),
                                         (int32_t)measurements_x.size(), K3DOM_MEM_HOST),
              "initializeParticles");
    }
    /* DOM::gridCellOccupancyUpdate (K3DOM: src/k3dom/dom.cu:79-94 with dt; DS:
     * src/dsphdmib/dom.cu:84-94 without, the overload below; dt is unused there). */
    void gridCellOccupancyUpdate(float dt, const std::vector<float>& measurements_x,
                                 const std::vector<float>& measurements_y, const std::vector<float>& measurements_z) {
        points(measurements_x, measurements_y, measurements_z);
        stage(k3dom_grid_cell_occupancy_update(h_, dt, measurements_x.data(), measurements_y.data(),
                                               measurements_z.data(), (int32_t)measurements_x.size(),
                                               K3DOM_MEM_HOST),
              "gridCellOccupancyUpdate");
    }
    void gridCellOccupancyUpdate(const std::vector<float>& measurements_x, const std::vector<float>& measurements_y,
                                 const std::vector<float>& measurements_z) {
        gridCellOccupancyUpdate(0.0f, measurements_x, measurements_y, measurements_z);
    }
};

}  // namespace dom

#endif  // K3DOM_B200_HPP
