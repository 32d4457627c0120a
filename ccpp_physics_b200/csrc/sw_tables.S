/* Embeds the RRTMG-SW coefficient blob (radsw_datatb.f DATA, extracted by
   ccpp_physics_b200/data/extract_sw_tables.py) in the shared library. */
        .section .rodata
        .balign 64
        .global rrtmg_sw_tables_blob
        .type rrtmg_sw_tables_blob, @object
rrtmg_sw_tables_blob:
        .incbin "rrtmg_sw_tables.bin"
        .global rrtmg_sw_tables_blob_end
rrtmg_sw_tables_blob_end:
        .byte 0
        .section .note.GNU-stack,"",@progbits
