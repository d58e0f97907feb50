// params.cpp -- node defaults, the flat YAML subset of config/*.yaml, and the unit
// conversions the ROS nodes apply before constructing dom::DOM.
//
// K3DOM node: defaults at src/k3dom/k3dom_node.cpp:219-258, rosparam reads :260-299,
// conversions :344-368. DS-PHD/MIB node: defaults dsphdmib_node.cpp:205-247, reads :249-290,
// conversions :330-356. yaml-cpp is not used; the config files are flat `key: value` maps.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "../../include/k3dom_b200.h"

namespace {

struct NodeValues {
    std::map<std::string, double> v;
    double get(const char* k) const { return v.at(k); }
};

NodeValues node_defaults(k3dom_variant variant) {
    NodeValues n;
    auto& v = n.v;
    const bool ds = variant == K3DOM_VARIANT_DSPHDMIB;
    v["resolution"] = 0.1f;
    v["ds_resolution"] = 0.1f;
    v["free_thresh"] = 0.3f;
    v["occupied_thresh"] = 0.7f;
    v["valid_thresh"] = ds ? 0.1f : 1.0f;
    v["min_z"] = 0.0f;
    v["max_z"] = 0.0f;
    v["min_var"] = 0.0f;
    v["max_var"] = 0.0f;
    v["map_pub_freq"] = 5;
    v["imu_pose_offset"] = 0.0f;
    v["size"] = 10.0f;
    v["size_z"] = 5.0f;
    v["mass_scale"] = 3.0f;
    v["meas_occ_stddev"] = 0.6f;
    v["do_eval"] = 0;
    v["map_vis_mode"] = 0;
    v["sensor_off_x"] = 0.0f;
    v["sensor_off_y"] = 0.0f;
    v["sensor_off_z"] = 0.0f;
    v["map_shift_thresh"] = 1.0f;
    v["particle_count"] = (float)(3 * static_cast<int>(10e6));
    v["new_born_particle_count"] = (float)(3 * static_cast<int>(10e5));
    v["persistence_prob"] = 0.99f;
    v["stddev_process_noise_position"] = 0.1f;
    v["stddev_process_noise_velocity"] = 1.0f;
    v["birth_prob"] = 0.02f;
    v["stddev_velocity"] = 1.0f;
    v["init_max_velocity"] = 5.0f;
    v["particle_min_vel"] = ds ? 0.0f : 1.0f;
    v["sigma"] = 1.0f;
    v["ls"] = 1.0f;
    v["gamma"] = 0.9f;
    v["prior_free"] = ds ? 0.0f : 1.0f;
    v["prior_static"] = ds ? 0.0f : 1.0f;
    v["prior_dynamic"] = ds ? 0.0f : 1.0f;
    v["prior_occ"] = 0.0f;
    return n;
}

// Keys each node reads with nh.param (the YAML key must match exactly).
const char* kK3domKeys[] = {"resolution", "ds_resolution", "free_thresh", "occupied_thresh", "valid_thresh",
                            "min_z", "max_z", "min_var", "max_var", "map_pub_freq", "imu_pose_offset", "size",
                            "size_z", "mass_scale", "do_eval", "map_vis_mode", "sensor_off_x", "sensor_off_y",
                            "sensor_off_z", "map_shift_thresh", "particle_count", "new_born_particle_count",
                            "persistence_prob", "stddev_process_noise_position", "stddev_process_noise_velocity",
                            "birth_prob", "stddev_velocity", "init_max_velocity", "particle_min_vel", "sigma", "ls",
                            "gamma", "prior_free", "prior_static", "prior_dynamic", "prior_occ", nullptr};
const char* kDsKeys[] = {"resolution", "ds_resolution", "free_thresh", "occupied_thresh", "min_z", "max_z",
                         "map_pub_freq", "imu_pose_offset", "size", "size_z", "mass_scale", "meas_occ_stddev",
                         "do_eval", "map_vis_mode", "sensor_off_x", "sensor_off_y", "sensor_off_z",
                         "map_shift_thresh", "particle_count", "new_born_particle_count", "persistence_prob",
                         "stddev_process_noise_position", "stddev_process_noise_velocity", "birth_prob",
                         "stddev_velocity", "init_max_velocity", "particle_min_vel", "prior_free", "prior_static",
                         "prior_dynamic", "prior_occ", nullptr};

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// Parses `key: value` lines; comments start at '#'. Returns false if the file is unreadable.
bool read_flat_yaml(const char* path, std::map<std::string, std::string>* out) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        size_t c = line.find(':');
        if (c == std::string::npos) continue;
        std::string k = trim(line.substr(0, c)), v = trim(line.substr(c + 1));
        if (k.empty() || v.empty()) continue;
        if (v.size() >= 2 && (v.front() == '"' || v.front() == '\'')) v = v.substr(1, v.size() - 2);
        (*out)[k] = v;
    }
    return true;
}

bool parse_number(const std::string& s, double* d) {
    if (s == "true" || s == "True") { *d = 1; return true; }
    if (s == "false" || s == "False") { *d = 0; return true; }
    char* end = nullptr;
    double x = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') return false;
    *d = x;
    return true;
}

// nh.param<float>(key, var, var): a readable number replaces the default. A value of the
// wrong type (e.g. `free_thresh: free_thresh`) leaves the default in place.
k3dom_status load(k3dom_variant variant, const char* method_yaml, const char* dataset_yaml, NodeValues* n) {
    *n = node_defaults(variant);
    std::map<std::string, std::string> kv;
    for (const char* path : {method_yaml, dataset_yaml}) {
        if (!path) continue;
        if (!read_flat_yaml(path, &kv)) return K3DOM_ERR_IO;
    }
    const bool ds = variant == K3DOM_VARIANT_DSPHDMIB;
    for (const char** k = ds ? kDsKeys : kK3domKeys; *k; ++k) {
        auto it = kv.find(*k);
        double d;
        if (it != kv.end() && parse_number(it->second, &d)) n->v[*k] = (float)d;
    }
    if (ds) {
        // dsphdmib_node.cpp:255 reads "occupied_thresh" into valid_thresh
        auto it = kv.find("occupied_thresh");
        double d;
        if (it != kv.end() && parse_number(it->second, &d)) n->v["valid_thresh"] = (float)d;
    }
    return K3DOM_OK;
}

void to_params(k3dom_variant variant, const NodeValues& n, k3dom_params* p) {
    std::memset(p, 0, sizeof(*p));
    const float res = (float)n.get("resolution");
    p->size = (float)n.get("size");
    p->size_z = (float)n.get("size_z");
    p->mass_scale = (float)n.get("mass_scale");
    p->resolution = res;
    p->particle_count = (int32_t)(float)n.get("particle_count");
    p->new_born_particle_count = (int32_t)(float)n.get("new_born_particle_count");
    p->persistence_prob = (float)n.get("persistence_prob");
    p->stddev_process_noise_position = (float)n.get("stddev_process_noise_position") / res;
    p->stddev_process_noise_velocity = (float)n.get("stddev_process_noise_velocity") / res;
    p->birth_prob = (float)n.get("birth_prob");
    p->stddev_velocity = (float)n.get("stddev_velocity") / res;
    p->init_max_velocity = (float)n.get("init_max_velocity") / res;
    p->particle_min_vel = (float)n.get("particle_min_vel") / res;
    p->sensor_off_x = (float)n.get("sensor_off_x");
    p->sensor_off_y = (float)n.get("sensor_off_y");
    p->sensor_off_z = (float)n.get("sensor_off_z");
    p->map_shift_thresh = static_cast<int>((float)n.get("map_shift_thresh") / res);
    p->prior_free = (float)n.get("prior_free");
    p->prior_static = (float)n.get("prior_static");
    p->prior_dynamic = (float)n.get("prior_dynamic");
    p->prior_occ = (float)n.get("prior_occ");
    if (variant == K3DOM_VARIANT_DSPHDMIB) {
        // the DS node leaves sigma/ls/gamma unset; they are unused by the variant
        p->sigma = 1.0f;
        p->ls = 1.0f;
        p->gamma = 0.9f;
        p->max_range = 50.0f;  // dsphdmib_node.cpp:346
        p->meas_occ_stddev = (float)n.get("meas_occ_stddev");
    } else {
        p->sigma = (float)n.get("sigma");
        p->ls = (float)n.get("ls");
        p->gamma = (float)n.get("gamma");
        // the K3DOM node leaves these unset; they are unused by the variant
        p->max_range = 50.0f;
        p->meas_occ_stddev = 0.6f;
    }
    p->seed = 0;
    p->max_points = 0;
}

}  // namespace

extern "C" {

k3dom_status k3dom_params_default(k3dom_variant variant, k3dom_params* out) {
    if (!out || (variant != K3DOM_VARIANT_K3DOM && variant != K3DOM_VARIANT_DSPHDMIB))
        return K3DOM_ERR_INVALID_ARGUMENT;
    to_params(variant, node_defaults(variant), out);
    return K3DOM_OK;
}

k3dom_status k3dom_params_from_yaml(k3dom_variant variant, const char* method_yaml, const char* dataset_yaml,
                                    k3dom_params* out) {
    if (!out || (variant != K3DOM_VARIANT_K3DOM && variant != K3DOM_VARIANT_DSPHDMIB))
        return K3DOM_ERR_INVALID_ARGUMENT;
    NodeValues n;
    k3dom_status s = load(variant, method_yaml, dataset_yaml, &n);
    if (s != K3DOM_OK) return s;
    to_params(variant, n, out);
    return K3DOM_OK;
}

k3dom_status k3dom_node_config_from_yaml(k3dom_variant variant, const char* method_yaml, const char* dataset_yaml,
                                         k3dom_node_config* out) {
    if (!out || (variant != K3DOM_VARIANT_K3DOM && variant != K3DOM_VARIANT_DSPHDMIB))
        return K3DOM_ERR_INVALID_ARGUMENT;
    NodeValues n;
    k3dom_status s = load(variant, method_yaml, dataset_yaml, &n);
    if (s != K3DOM_OK) return s;
    out->occupied_thresh = (float)n.get("occupied_thresh");
    out->valid_thresh = (float)n.get("valid_thresh");
    out->free_thresh = (float)n.get("free_thresh");
    out->min_z = (float)n.get("min_z");
    out->max_z = (float)n.get("max_z");
    out->min_var = (float)n.get("min_var");
    out->max_var = (float)n.get("max_var");
    out->ds_resolution = (float)n.get("ds_resolution");
    out->imu_pose_offset = (float)n.get("imu_pose_offset");
    out->map_pub_freq = (int32_t)n.get("map_pub_freq");
    out->map_vis_mode = (int32_t)n.get("map_vis_mode");
    out->do_eval = (int32_t)n.get("do_eval");
    return K3DOM_OK;
}

}  // extern "C"
