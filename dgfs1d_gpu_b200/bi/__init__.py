"""Binary-mixture solver pieces behind the plugin keys of dgfsBi1D."""
