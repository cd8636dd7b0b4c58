/*
 * libfyaml stand-in for the HigFlow host build and the oracle build.  Both
 * fill the solver parameters directly (higflow_b200/host/hf_host.c), so the
 * YAML readers compiled in from the reference are never called; each entry
 * point aborts if reached.
 */
#ifndef HF_ORACLE_LIBFYAML_SHIM_H
#define HF_ORACLE_LIBFYAML_SHIM_H
struct fy_document;
struct fy_parse_cfg;
struct fy_document *fy_document_build_from_file(const struct fy_parse_cfg *cfg, const char *file);
void fy_document_destroy(struct fy_document *fyd);
int fy_document_scanf(struct fy_document *fyd, const char *fmt, ...);
#endif
