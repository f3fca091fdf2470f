/* Embeds the glibc expf exception table (generated at build time by
   gen_expf_table) into the shared library. */
    .section .rodata
    .balign 16
    .global tamc_expf_blob_begin
    .global tamc_expf_blob_end
tamc_expf_blob_begin:
    .incbin EXPF_TABLE_BIN
tamc_expf_blob_end:
    .section .note.GNU-stack,"",@progbits
