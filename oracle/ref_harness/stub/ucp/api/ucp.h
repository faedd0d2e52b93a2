/* Opaque stand-ins for the UCX handle types named by the reference's
 * src/shmemc/ucx/pe.h team/context structs.  Nothing here is called: the
 * PE emulator replaces the UCX transport entirely. */
#ifndef PE_EMU_UCP_STUB_H
#define PE_EMU_UCP_STUB_H
typedef void *ucp_address_t;
typedef void *ucp_rkey_h;
typedef void *ucp_mem_h;
typedef void *ucp_worker_h;
typedef void *ucp_ep_h;
typedef void *ucp_context_h;
typedef void *ucp_config_t;
typedef int ucs_thread_mode_t;
typedef int ucs_status_t;
#endif
