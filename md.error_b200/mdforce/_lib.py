"""ctypes loader of libmdforce.so (the C ABI declared in include/mdforce.h).

The library is built in-tree by ``make -C md.error_b200/csrc``.  There is no
fallback: if the shared object is missing or cannot be loaded, importing
this module raises, so nothing can silently run on the CPU instead.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmdforce.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libmdforce.so not found at {LIB_PATH}; build it with "
        "`make -C md.error_b200/csrc` (nvcc, sm_100a)")

lib = C.CDLL(LIB_PATH)

vp = C.c_void_p
i32 = C.c_int
i64 = C.c_int64
u64 = C.c_uint64
f32 = C.c_float
f64 = C.c_double
P = C.POINTER


class DeviceView(C.Structure):
    """md_device_view: raw device pointers (caller's atom order)"""
    _fields_ = [("pos", C.c_void_p), ("charge", C.c_void_p)]


class LangevinParams(C.Structure):
    """md_langevin_params"""
    _fields_ = [("dt", f64), ("temperature", f64), ("gamma_t", f64),
                ("tau_p", f64), ("kappa_t", f64), ("p_ref", f64 * 3),
                ("npt_dirs", i32), ("seed", u64)]


class SimParams(C.Structure):
    """md_sim_params"""
    _fields_ = [("lv", LangevinParams), ("skin", f64), ("cell_size", f64),
                ("expansion", f64), ("nl_mode", i32), ("use_graph", i32),
                ("stats_every", i32), ("max_rcut", f64), ("integrator", i32), ("nhc_tau", f64),
                ("remove_com", i32), ("spme", C.c_void_p)]


_SIGS = {
    "md_last_error_message": (C.c_char_p, []),
    "md_version": (C.c_char_p, []),
    "md_device_count": (i32, [P(i32)]),
    "md_system_create": (i32, [P(vp), i32, P(f64), P(f64), P(f64), P(i32), P(f64), P(f64), i32, i32]),
    "md_system_destroy": (i32, [vp]),
    "md_system_set_stream": (i32, [vp, vp]),
    "md_system_synchronize": (i32, [vp]),
    "md_system_num_atoms": (i32, [vp, P(i32)]),
    "md_system_set_positions": (i32, [vp, P(f64)]),
    "md_system_get_positions": (i32, [vp, P(f64)]),
    "md_system_get_unwrapped_positions": (i32, [vp, P(f64)]),
    "md_system_set_velocities": (i32, [vp, P(f64)]),
    "md_system_get_velocities": (i32, [vp, P(f64)]),
    "md_system_get_forces": (i32, [vp, P(f64)]),
    "md_system_get_box": (i32, [vp, P(f64)]),
    "md_system_set_box": (i32, [vp, P(f64)]),
    "md_system_set_rcut": (i32, [vp, P(f32)]),
    "md_system_get_rcut": (i32, [vp, P(f32)]),
    "md_system_normalize": (i32, [vp]),
    "md_system_read_stats": (i32, [vp, P(f64)]),
    "md_system_read_stats_async": (i32, [vp, P(f64)]),
    "md_system_clear_stats": (i32, [vp]),
    "md_cell_list_create": (i32, [P(vp), vp, f64, i32, i32]),
    "md_cell_list_destroy": (i32, [vp]),
    "md_cell_list_rebuild": (i32, [vp, vp]),
    "md_cell_list_get_ncell": (i32, [vp, P(i32)]),
    "md_cell_list_get_cell_index": (i32, [vp, vp, P(C.c_uint32)]),
    "md_nlist_create": (i32, [P(vp), vp, f64, f64, f64, i32]),
    "md_nlist_destroy": (i32, [vp]),
    "md_nlist_rebuild": (i32, [vp, vp, vp]),
    "md_nlist_fit": (i32, [vp, vp, vp]),
    "md_nlist_capacity": (i32, [vp, P(i32)]),
    "md_nlist_max_displacement": (i32, [vp, vp, P(f64)]),
    "md_nlist_sum_neighbor": (i32, [vp, vp, P(i64)]),
    "md_nlist_get": (i32, [vp, vp, P(C.c_int32), P(C.c_int32)]),
    "md_engine_create": (i32, [P(vp), vp]),
    "md_engine_destroy": (i32, [vp]),
    "md_engine_register_lj": (i32, [vp, f64, f64, f64]),
    "md_engine_register_bonded": (i32, [vp, i32]),
    "md_engine_clear_forces": (i32, [vp, vp]),
    "md_engine_apply_nonbonded": (i32, [vp, vp, vp, i32]),
    "md_engine_finish_nonbonded_stats": (i32, [vp, vp]),
    "md_engine_apply_bonded": (i32, [vp, vp]),
    "md_engine_set_bonds": (i32, [vp, i32, P(i32), P(i32), P(f64)]),
    "md_engine_register_lj_pair": (i32, [vp, i32, i32, f64, f64, f64]),
    "md_engine_register_nb_pair": (i32, [vp, i32, i32, i32, P(f64)]),
    "md_system_set_types": (i32, [vp, P(i32)]),
    "md_system_get_types": (i32, [vp, P(i32)]),
    "md_engine_set_angles": (i32, [vp, i32, P(i32), P(i32), P(f64)]),
    "md_engine_set_exclusions": (i32, [vp, i32, P(i32)]),
    "md_nlist_apply_exclusions": (i32, [vp, vp]),
    "md_assign_rcut": (i32, [vp, P(f32), i32, i32, i32]),
    "md_set_rcut_uniform": (i32, [vp, f32]),
    "md_vv_step1": (i32, [vp, f64]),
    "md_vv_step2": (i32, [vp, f64, i32]),
    "md_langevin_setup": (i32, [vp, P(LangevinParams)]),
    "md_langevin_step1": (i32, [vp, vp]),
    "md_langevin_step2": (i32, [vp]),
    "md_langevin_get_state": (i32, [vp, P(f64), P(f64)]),
    "md_sim_create": (i32, [P(vp), vp, vp, P(SimParams)]),
    "md_sim_destroy": (i32, [vp]),
    "md_sim_run": (i32, [vp, i32]),
    "md_sim_counters": (i32, [vp, P(i64), P(i64), P(i32)]),
    "md_sim_uses_conditional_graph": (i32, [vp, P(i32)]),
    "md_sim_rebuild_kind": (i32, [vp, P(i32)]),
    "md_sim_set_rebuild_kind": (i32, [vp, i32]),
    "md_check_grid_barrier": (i32, [vp, i32, f64, P(i32)]),
    "md_engine_register_coulomb": (i32, [vp, f64]),
    "md_spme_create": (i32, [P(vp), vp, P(i32), i32, f64, i32]),
    "md_spme_destroy": (i32, [vp]),
    "md_spme_apply": (i32, [vp, vp, i32]),
    "md_spme_get_mesh": (i32, [vp, P(f64)]),
    "md_spme_energy_grad": (i32, [vp, vp, P(f64), P(f64), P(f64), P(f64), P(f64)]),
    "md_spme_energy_grad_device": (i32, [vp, vp, vp, vp, vp, vp]),
    "md_system_set_device_view": (i32, [vp, P(DeviceView)]),
    "md_hspme_create": (i32, [P(vp), i32, P(i32), P(f64), f64, f64, i32, i32, i32]),
    "md_hspme_destroy": (i32, [vp]),
    "md_hspme_num_coeffs": (i32, [vp, P(i32)]),
    "md_hspme_energy": (i32, [vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp]),
    "md_hspme_force_error": (i32, [vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp]),
    "md_spme_get_influence": (i32, [vp, P(f64)]),
    "md_spme_self_correction": (i32, [vp, vp]),
    "md_system_set_charges": (i32, [vp, P(f64)]),
    "md_system_get_charges": (i32, [vp, P(f64)]),
    "md_system_set_masses": (i32, [vp, P(f64)]),
    "md_system_get_masses": (i32, [vp, P(f64)]),
    "md_ewald_self_energy": (i32, [vp, f64, P(f64)]),
    "md_ewald_exact": (i32, [vp, P(i32), f64, P(f64), i32]),
    "md_error_estimate_pme": (i32, [vp, P(i32), f64, f64, P(f64), P(f64)]),
    "md_error_estimate_spme_ik": (i32, [vp, P(i32), i32, f64, P(f64)]),
    "md_error_estimate_spme_ik_noalloc": (i32, [vp, P(i32), i32, f64, P(f64)]),
    "md_choose_beta": (i32, [vp, f64, f64, P(f64)]),
    "md_choose_spme_params": (i32, [vp, f64, i32, f64, i32, P(f64), P(i32), P(f64), P(f64)]),
    "md_sim_attach_adapt_rcut": (i32, [vp, vp, i32, i32, f64, i32]),
    "md_arc_create": (i32, [P(vp), vp, f64, f64, f64, f64]),
    "md_arc_destroy": (i32, [vp]),
    "md_arc_get_dims": (i32, [vp, P(i32), P(i32)]),
    "md_arc_deposit": (i32, [vp, vp]),
    "md_arc_clear_profile": (i32, [vp]),
    "md_arc_set_profile": (i32, [vp, P(f64)]),
    "md_arc_get_profile": (i32, [vp, P(f64)]),
    "md_arc_update": (i32, [vp, f64, i32]),
    "md_arc_get_error": (i32, [vp, P(f64)]),
    "md_arc_get_rcut": (i32, [vp, P(f64), P(i32), P(f64)]),
    "md_arc_get_tables": (i32, [vp, P(f64), P(f64), P(f64)]),
    "md_arc_assign": (i32, [vp, vp]),
    "md_arc_pressure_correction": (i32, [vp, vp, P(f64)]),
    "md_synth_fcc": (i32, [i32, i32, i32, P(f64), f64, u64, P(f64)]),
    "md_gro_count": (i32, [C.c_char_p, P(i32)]),
    "md_gro_read": (i32, [C.c_char_p, i32, P(i32), P(C.c_char), P(C.c_char), P(i32), P(f64), P(f64), P(f64)]),
    "md_gro_write": (i32, [C.c_char_p, C.c_char_p, i32, P(i32), P(C.c_char), P(C.c_char), P(i32), P(f64),
                           P(f64), P(f64)]),
    "md_synth_slab": (i32, [i32, i32, P(f64), i32, f64, f64, f64, u64, P(f64)]),
    "md_synth_maxwell": (i32, [i32, P(f64), f64, u64, P(f64)]),
    "md_synth_charges": (i32, [i32, u64, P(f64)]),
    "md_nhc_create": (i32, [P(vp), vp, f64, f64, i32]),
    "md_nhc_destroy": (i32, [vp]),
    "md_nhc_operator_L": (i32, [vp, vp, f64, i32]),
    "md_nhc_step1": (i32, [vp, vp, vp, f64]),
    "md_nhc_step2": (i32, [vp, vp, f64]),
    "md_nhc_get_state": (i32, [vp, P(f64)]),
    "md_sim_get_nhc_state": (i32, [vp, P(f64)]),
    "md_nhc_npt_create": (i32, [P(vp), vp, f64, f64, f64, f64, f64]),
    "md_nhc_npt_destroy": (i32, [vp]),
    "md_nhc_npt_operator_L_CP": (i32, [vp, vp, f64]),
    "md_nhc_npt_operator_L_v": (i32, [vp, vp, f64]),
    "md_nhc_npt_operator_L_r": (i32, [vp, vp, f64]),
    "md_nhc_npt_operator_L_box": (i32, [vp, vp, f64]),
    "md_nhc_npt_get_state": (i32, [vp, P(f64)]),
    "md_errmap_create": (i32, [P(vp), P(i32), P(f64), f64, i32, i32]),
    "md_errmap_destroy": (i32, [vp]),
    "md_errmap_create_dir": (i32, [P(vp), P(i32), P(f64), f64, f64, i32]),
    "md_errmap_create_ana": (i32, [P(vp), P(i32), P(f64), f64, i32, i32]),
    "md_errmap_self_error": (i32, [vp, P(f64)]),
    "md_errmap_ana_fconv": (i32, [vp, i32, P(f64)]),
    "md_errmap_mean_force": (i32, [vp, f64, P(f64)]),
    "md_errmap_set_profile": (i32, [vp, P(f64), P(f64)]),
    "md_errmap_deposit": (i32, [vp, vp]),
    "md_errmap_get_profile": (i32, [vp, P(f64), P(f64)]),
    "md_errmap_compute": (i32, [vp, f64, P(f64), P(f64)]),
    "md_ikerr_create":(i32, [P(vp), P(i32), P(f64), f64, f64, i32, i32, i32, i32, f64, f64, i32]),
    "md_ikerr_destroy": (i32, [vp]),
    "md_ikerr_num_coeffs": (i32, [vp, P(i32)]),
    "md_ikerr_evaluate": (i32, [vp, i32, P(f64), P(f64), P(f64)]),
    "md_ikerr_evaluate_device": (i32, [vp, i32, vp, vp, vp, vp]),
    "md_ikerr_get_hats": (i32, [vp, i32, P(f64), P(f64)]),
    "md_ikerr_get_weights": (i32, [vp, i32, P(f64)]),
    "md_fcorr_create": (i32, [P(vp), vp, f64, f64]),
    "md_fcorr_destroy": (i32, [vp]),
    "md_fcorr_get_dims": (i32, [vp, P(i32)]),
    "md_fcorr_deposit": (i32, [vp, vp]),
    "md_fcorr_clear_profile": (i32, [vp]),
    "md_fcorr_set_profile": (i32, [vp, P(f64)]),
    "md_fcorr_get_profile": (i32, [vp, P(f64)]),
    "md_fcorr_update": (i32, [vp]),
    "md_fcorr_zero": (i32, [vp]),
    "md_fcorr_get_field": (i32, [vp, P(f64), P(f64)]),
    "md_fcorr_assign": (i32, [vp, vp]),
    "md_fcorr_get_values": (i32, [vp, P(f64)]),
    "md_engine_set_force_correction": (i32, [vp, vp]),
    "md_sim_attach_force_corr": (i32, [vp, vp, i32, i32, i32]),
    "md_sim_set_stats_ring": (i32, [vp, P(f64), i32]),
}


def _declare(sigs):
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


_declare(_SIGS)
EXPORTED = tuple(_SIGS)
