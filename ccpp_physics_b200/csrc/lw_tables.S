/* Embeds the RRTMG-LW coefficient blob (radlw_datatb.f DATA, extracted by
   ccpp_physics_b200/data/extract_tables.py) in the shared library. */
        .section .rodata
        .balign 64
        .global rrtmg_lw_tables_blob
        .type rrtmg_lw_tables_blob, @object
rrtmg_lw_tables_blob:
        .incbin "rrtmg_lw_tables.bin"
        .global rrtmg_lw_tables_blob_end
rrtmg_lw_tables_blob_end:
        .byte 0
        .section .note.GNU-stack,"",@progbits
