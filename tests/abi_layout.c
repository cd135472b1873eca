/* Prints the size and field offsets of the C-ABI structs of include/jfb200.h
 * so that tests/test_abi.py can compare them with the ctypes mirrors. */
#include <stddef.h>
#include <stdio.h>

#include "jfb200.h"

#define F(T, f) printf("%s.%s %zu\n", #T, #f, offsetof(T, f))

int main(void) {
  printf("jfb_kmm_config %zu\n", sizeof(jfb_kmm_config));
  F(jfb_kmm_config, nx); F(jfb_kmm_config, family); F(jfb_kmm_config, x_lo);
  F(jfb_kmm_config, ly); F(jfb_kmm_config, pad_y); F(jfb_kmm_config, nu);
  F(jfb_kmm_config, dt); F(jfb_kmm_config, u_wall); F(jfb_kmm_config, precision);
  F(jfb_kmm_config, nonlinear_form); F(jfb_kmm_config, time_integrator);
  printf("jfb_kmm_state %zu\n", sizeof(jfb_kmm_state));
  F(jfb_kmm_state, u0); F(jfb_kmm_state, g); F(jfb_kmm_state, nonlinear_old);
  F(jfb_kmm_state, nonlinear_older); F(jfb_kmm_state, solution_old);
  F(jfb_kmm_state, solution_older); F(jfb_kmm_state, history_steps);
  printf("jfb_kmm_info %zu\n", sizeof(jfb_kmm_info));
  F(jfb_kmm_info, n_pencils); F(jfb_kmm_info, algorithmic_bytes); F(jfb_kmm_info, my);
  F(jfb_kmm_info, mz);
  printf("jfb_mhd_state %zu\n", sizeof(jfb_mhd_state));
  F(jfb_mhd_state, flow); F(jfb_mhd_state, A); F(jfb_mhd_state, nonlinear_A_old);
  F(jfb_mhd_state, nonlinear_A_older); F(jfb_mhd_state, A_old); F(jfb_mhd_state, A_older);
  printf("jfb_mhd_params %zu\n", sizeof(jfb_mhd_params));
  F(jfb_mhd_params, eta); F(jfb_mhd_params, omega); F(jfb_mhd_params, b0);
  printf("jfb_tps_config %zu\n", sizeof(jfb_tps_config));
  F(jfb_tps_config, ndim); F(jfb_tps_config, n); F(jfb_tps_config, x_lo);
  F(jfb_tps_config, l); F(jfb_tps_config, pad); F(jfb_tps_config, family);
  printf("jfb_kmm_variant %zu\n", sizeof(jfb_kmm_variant));
  F(jfb_kmm_variant, pencil); F(jfb_kmm_variant, tc_velocity); F(jfb_kmm_variant, replicas);
  return 0;
}
