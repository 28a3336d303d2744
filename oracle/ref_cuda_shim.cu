// ref_cuda_shim.cu - C entry points around the reference's own GPU engine,
// compiled into oracle/_ref/libref_cuda.so from a copy of cuda_engine.cu that
// build_ref.py makes headless (the GL-interop include and the one GL buffer
// registration call removed) and whose opening test reads the variable
// ref_theta_sq in place of the literal 1.0f (cuda_engine.cu:143).  With
// ref_theta_sq = 1 the code is the reference's, unchanged.
//
// TEST/BASELINE INFRASTRUCTURE ONLY: GPU parity tests and the bench's
// reference-GPU timing call it; the engine never does.
//
// ref_cuda_step_device runs the kernel sequence of cuda_physics_step
// (cuda_engine.cu:394-424) without the output transpose and copy, timed
// with CUDA events; ref_cuda_step calls cuda_physics_step itself.
#include "cuda_engine_headless.cu"

extern "C" {

int ref_cuda_init(int n) { return cuda_init(n) ? 0 : -1; }

void ref_cuda_cleanup(void) { cuda_cleanup(); }

void ref_cuda_upload(const Star* host, int n) { cuda_upload_initial_stars(host, n); }

int ref_cuda_set_theta(float theta) {
    const float t2 = theta * theta;
    return cudaMemcpyToSymbol(ref_theta_sq, &t2, sizeof(float)) == cudaSuccess ? 0 : -1;
}

float ref_cuda_step(Star* host, int n, float G, float eps2, float dt, float lo, float hi) {
    return cuda_physics_step(host, n, G, eps2, dt, lo, hi, false);
}

// cuda_engine.cu:389-424 (everything but the output), returns milliseconds.
float ref_cuda_step_device(int n, float G, float eps2, float dt, float lo, float hi) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int threads = 256;
    const int blocks_n = (n + threads - 1) / threads;
    const int blocks_n1 = (n - 1 + threads - 1) / threads;
    cudaEventRecord(a);
    cudaMemset(d_max_accel_int, 0, sizeof(int));
    compute_morton_and_indices_kernel<<<blocks_n, threads>>>(d_x, d_y, d_z, d_morton_keys, d_indices, n, lo, hi);
    cub::DeviceRadixSort::SortPairs(d_temp_storage, temp_storage_bytes, d_morton_keys, d_morton_keys_out,
                                    d_indices, d_indices_out, n);
    apply_sorted_indices_kernel<<<blocks_n, threads>>>(
        d_indices_out, d_x, d_y, d_z, d_vx, d_vy, d_vz, d_mass, d_r, d_g, d_b, d_type, d_x_alt, d_y_alt,
        d_z_alt, d_vx_alt, d_vy_alt, d_vz_alt, d_mass_alt, d_r_alt, d_g_alt, d_b_alt, d_type_alt, n);
    swap_ptr(d_x, d_x_alt);
    swap_ptr(d_y, d_y_alt);
    swap_ptr(d_z, d_z_alt);
    swap_ptr(d_vx, d_vx_alt);
    swap_ptr(d_vy, d_vy_alt);
    swap_ptr(d_vz, d_vz_alt);
    swap_ptr(d_mass, d_mass_alt);
    swap_ptr(d_r, d_r_alt);
    swap_ptr(d_g, d_g_alt);
    swap_ptr(d_b, d_b_alt);
    swap_ptr(d_type, d_type_alt);
    init_internal_nodes_kernel<<<blocks_n1, threads>>>(n, d_bvh_nodes_tr, d_bvh_nodes_bd);
    init_leaves_kernel<<<blocks_n, threads>>>(n, d_bvh_nodes_tr, d_bvh_nodes_bd, d_x, d_y, d_z, d_mass);
    build_radix_tree_kernel<<<blocks_n1, threads>>>(n, d_morton_keys_out, d_bvh_nodes_tr, d_bvh_nodes_bd);
    cudaDeviceSynchronize();
    aggregate_bvh_kernel<<<blocks_n, threads>>>(n, d_bvh_nodes_tr, d_bvh_nodes_bd);
    cudaDeviceSynchronize();
    query_gravity_bvh_kernel<<<blocks_n, threads>>>(d_x, d_y, d_z, d_mass, n, d_bvh_nodes_tr, G, eps2,
                                                    d_accels, d_max_accel_int);
    integrate_kernel<<<blocks_n, threads>>>(d_x, d_y, d_z, d_vx, d_vy, d_vz, d_r, d_g, d_b, d_type,
                                            d_accels, dt, n);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

// Milliseconds of the walk kernel alone on the current tree and positions.
float ref_cuda_time_walk(int n, float G, float eps2) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int threads = 256;
    cudaEventRecord(a);
    query_gravity_bvh_kernel<<<(n + threads - 1) / threads, threads>>>(d_x, d_y, d_z, d_mass, n, d_bvh_nodes_tr,
                                                                      G, eps2, d_accels, d_max_accel_int);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

// Copy an internal array to host.  which: 0 sorted keys (u64 n), 1 sorted
// indices (i32 n), 2 traverse nodes (32 B, 2n-1), 3 build nodes (32 B, 2n-1),
// 4 accels (float3 n), 5 SoA x,y,z,vx,vy,vz,mass (7 floats x n, in that
// order), 6 SoA r,g,b,type (4 bytes x n).
int ref_cuda_read(int which, void* host, int n) {
    cudaDeviceSynchronize();
    cudaError_t e = cudaSuccess;
    switch (which) {
        case 0: e = cudaMemcpy(host, d_morton_keys_out, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost); break;
        case 1: e = cudaMemcpy(host, d_indices_out, sizeof(int) * n, cudaMemcpyDeviceToHost); break;
        case 2: e = cudaMemcpy(host, d_bvh_nodes_tr, sizeof(BvhNodeTraverse) * (2 * n - 1), cudaMemcpyDeviceToHost); break;
        case 3: e = cudaMemcpy(host, d_bvh_nodes_bd, sizeof(BvhNodeBuild) * (2 * n - 1), cudaMemcpyDeviceToHost); break;
        case 4: e = cudaMemcpy(host, d_accels, sizeof(float3) * n, cudaMemcpyDeviceToHost); break;
        case 5: {
            float* out = static_cast<float*>(host);
            float* src[7] = {d_x, d_y, d_z, d_vx, d_vy, d_vz, d_mass};
            for (int k = 0; k < 7 && e == cudaSuccess; ++k)
                e = cudaMemcpy(out + (size_t)k * n, src[k], sizeof(float) * n, cudaMemcpyDeviceToHost);
            break;
        }
        case 6: {
            uint8_t* out = static_cast<uint8_t*>(host);
            uint8_t* src[4] = {d_r, d_g, d_b, d_type};
            for (int k = 0; k < 4 && e == cudaSuccess; ++k)
                e = cudaMemcpy(out + (size_t)k * n, src[k], n, cudaMemcpyDeviceToHost);
            break;
        }
        default: return -1;
    }
    return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
