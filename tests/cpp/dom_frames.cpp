// Drives dom::DOM (include/k3dom_b200.hpp) through a few frames the way the reference's ROS node
// drives its own dom::DOM (src/k3dom/k3dom_node.cpp:64-97,129-184): updatePose, updateGrid with
// three coordinate vectors, a cudaMemcpy of grid_cell_array into grid_cell_array_host, and the
// /map_data cloud built from the GridCell helpers and indexToCoord*.
//
//   dom_frames <dir>
//
// <dir> holds params.bin (a k3dom_params), frames.txt ("n" then one "t x y z npoints" line per
// frame) and scan<f>.bin (npoints x 3 floats). Writes cells.bin (the 68-byte records after the
// last frame), mappoints_node.bin (publish_mapdata's formula on those records) and
// mappoints_lib.bin (k3dom_get_mappoints), then prints "ok <grid_cell_count>".
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "k3dom_b200.hpp"

static std::vector<char> slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot read " + path);
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

static void spill(const std::string& path, const void* data, size_t bytes) {
    std::ofstream f(path, std::ios::binary);
    f.write(static_cast<const char*>(data), (std::streamsize)bytes);
    if (!f) throw std::runtime_error("cannot write " + path);
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <dir>\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    try {
        std::vector<char> pb = slurp(dir + "/params.bin");
        dom::DOM::Params params;
        if (pb.size() != sizeof(k3dom_params)) throw std::runtime_error("params.bin size");
        std::memcpy(static_cast<k3dom_params*>(&params), pb.data(), sizeof(k3dom_params));
        dom::DOM grid_map(params);

        std::ifstream frames(dir + "/frames.txt");
        int n_frames = 0;
        frames >> n_frames;
        for (int f = 0; f < n_frames; ++f) {
            float t, x, y, z;
            int n;
            frames >> t >> x >> y >> z >> n;
            std::vector<char> raw = slurp(dir + "/scan" + std::to_string(f) + ".bin");
            const float* xyz = reinterpret_cast<const float*>(raw.data());
            std::vector<float> pc_x(n), pc_y(n), pc_z(n);
            for (int i = 0; i < n; ++i) {
                pc_x[i] = xyz[3 * i];
                pc_y[i] = xyz[3 * i + 1];
                pc_z[i] = xyz[3 * i + 2];
            }
            grid_map.updatePose(x, y, z);
            grid_map.updateGrid(t, pc_x, pc_y, pc_z);
        }

        // the node's readback (k3dom_node.cpp:131-132)
        if (cudaMemcpy(grid_map.grid_cell_array_host, grid_map.grid_cell_array,
                       grid_map.grid_cell_count * sizeof(dom::GridCell), cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("cudaMemcpy of grid_cell_array");
        spill(dir + "/cells.bin", grid_map.grid_cell_array_host, grid_map.grid_cell_count * sizeof(dom::GridCell));

        // publish_mapdata (k3dom_node.cpp:161-184)
        const float res = grid_map.getResolution();
        std::vector<dom::MapPoint> pts((size_t)grid_map.grid_cell_count);
        for (int i = 0; i < grid_map.grid_cell_count; ++i) {
            const dom::GridCell& c = grid_map.grid_cell_array_host[i];
            dom::MapPoint& pt = pts[(size_t)i];
            pt.x = grid_map.indexToCoordX(i);
            pt.y = grid_map.indexToCoordY(i);
            pt.z = grid_map.indexToCoordZ(i);
            pt.v_x = c.mean_x_vel * res;
            pt.v_y = c.mean_y_vel * res;
            pt.v_z = c.mean_z_vel * res;
            pt.occ_val = c.occ_mean();
            pt.dyn_val = c.dyn_mean();
            pt.eval_aug = c.total_mass();
            pt.dyn_aug = 1.1f;
        }
        spill(dir + "/mappoints_node.bin", pts.data(), pts.size() * sizeof(dom::MapPoint));
        std::vector<dom::MapPoint> lib = grid_map.mapPoints();
        spill(dir + "/mappoints_lib.bin", lib.data(), lib.size() * sizeof(dom::MapPoint));
        std::printf("ok %d\n", grid_map.grid_cell_count);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
